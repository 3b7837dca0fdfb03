"""FDMAP input files (.in namelists + binary side files) for the benchmark
configurations.  The texts use only FDMAP's own input vocabulary, so the same
files drive FDMAP itself, the host initialisation here and the CPU oracle.

Units follow FDMAP: km, s, m/s, MPa, g/cm^3, km/s (2670 kg/m^3 -> 2.67,
3464 m/s -> 3.464, 25 m -> 0.025).

  antiplane_pulse      mode III SH pulse, one Cartesian block          (config "c1")
  rupture_sw           mode II slip-weakening rupture, two blocks      (config "c2")
  rough_fault_rs       mode II rate-and-state on a rough fault         (config "c3")
  heterogeneous_ricker mode III heterogeneous medium, Ricker point force (config "c5")
  ensemble_instance    mode II rate-and-state, planar fault, von Karman prestress (config "c4")
  pml_pulse            mode II P-SV pulse in a block with a perfectly matched layer
  gaussian_forcing     mode III long-wave forcing, Gaussian in space and time (problem='Forcing')
  write_forcing_file   a forcing file sampling the same Gaussian, one frame per step
"""
from __future__ import annotations

from pathlib import Path

import numpy as np


def _f(x: float) -> str:
    """Fortran double literal."""
    return repr(float(x)).replace("e", "d") if "e" in repr(float(x)) else repr(float(x)) + "d0"


def _operator(cdiss: float) -> str:
    """operator_list of a block: artificial dissipation coefficient (domain.f90:89)."""
    return f"&operator_list Cdiss={_f(cdiss)} /\n" if cdiss > 0 else ""


def antiplane_pulse(n: int = 201, L: float = 10.0, nt: int = 501, rk: int = 4, cfl: float = 0.5,
                    fd: str = "SBP4", sigma: float = 0.5, amp: float = 1.0, cdiss: float = 0.0) -> str:
    """Mode III SH wave from a Gaussian velocity pulse at the centre of an L x L km
    block of n x n nodes, absorbing SAT boundaries on all sides; optional
    artificial dissipation `cdiss`."""
    c = 0.5 * L
    return f"""&problem_list name='antiplane_pulse', nt={nt}, CFL={_f(cfl)}, RKorder={rk} /
&domain_list mode=3, FDmethod='{fd}', nblocks_x=1, nblocks_y=1 /
!---BLOCK1---
&grid_list nx={n}, ny={n}, LB=0d0,0d0, LT=0d0,{_f(L)}, RB={_f(L)},0d0, RT={_f(L)},{_f(L)} /
&boundaries_list bcL='absorbing', bcR='absorbing', bcB='absorbing', bcT='absorbing' /
{_operator(cdiss)}&material_list rho=2.67d0, cs=3.464d0 /
&fields_list P5%shape='gaussian', P5%x0={_f(c)}, P5%y0={_f(c)}, P5%Lx={_f(sigma)}, P5%Ly={_f(sigma)}, P5%vz={_f(amp)} /
"""


def _pml(pmlx: bool, pmly: bool, npow: float, sigma: float, kappa: float, lo: float, hi: float) -> str:
    """pml_list of a block (material.f90:152-222): the layer starts at x, y = lo and hi."""
    t = "T" if pmlx else "F"
    u = "T" if pmly else "F"
    return (f"&pml_list pmlx={t}, pmly={u}, n={_f(npow)}, sigma={_f(sigma)}, kappa={_f(kappa)},\n"
            f"  mx={_f(lo)}, px={_f(hi)}, my={_f(lo)}, py={_f(hi)} /\n")


def pml_pulse(n: int = 201, L: float = 10.0, nt: int = 401, rk: int = 4, cfl: float = 0.5, fd: str = "SBP4",
              width: float = 1.5, npow: float = 2.0, R: float = 1e-3, kappa: float = 0.0, pmlx: bool = True,
              pmly: bool = True, bc: str = "free", sigma: float | None = None, cdiss: float = 0.0,
              mode: int = 2) -> str:
    """Mode II P-SV waves from a Gaussian pulse (vx and sxx) near the centre of an
    L x L km block of n x n nodes with a perfectly matched layer of `width` km
    along every side: damping sigma*d^npow at distance d into the layer, sigma
    chosen for a reflection coefficient R at normal incidence
    (sigma_max = (npow+1)*cp*ln(1/R)/(2*width)) unless given.  `bc` applies to
    all four sides ('free' reflects everything the layer lets through)."""
    cp = 6.0
    if sigma is None:
        smax = (npow + 1.0) * cp * np.log(1.0 / R) / (2.0 * width)
        sigma = smax / width ** npow if npow > 0 else smax
    c = 0.5 * L
    f = ("&fields_list P5%shape='gaussian', P5%x0={x0}, P5%y0={y0}, P5%Lx=0.4d0, P5%Ly=0.4d0, "
         "P5%vx=1d0, P5%sxx=2d0 /\n").format(x0=_f(c - 0.3), y0=_f(c + 0.2))
    if mode == 3:
        f = f"&fields_list P5%shape='gaussian', P5%x0={_f(c)}, P5%y0={_f(c)}, P5%Lx=0.4d0, P5%Ly=0.4d0, P5%vz=1d0 /\n"
    return f"""&problem_list name='pml_pulse', nt={nt}, CFL={_f(cfl)}, RKorder={rk} /
&domain_list mode={mode}, FDmethod='{fd}', nblocks_x=1, nblocks_y=1 /
!---BLOCK1---
&grid_list nx={n}, ny={n}, LB=0d0,0d0, LT=0d0,{_f(L)}, RB={_f(L)},0d0, RT={_f(L)},{_f(L)} /
&boundaries_list bcL='{bc}', bcR='{bc}', bcB='{bc}', bcT='{bc}' /
{_operator(cdiss)}&material_list rho=2.67d0, cs=3.464d0, cp={_f(cp)} /
{f}{_pml(pmlx, pmly, npow, sigma, kappa, width, L - width)}"""


def gaussian_forcing(n: int = 101, L: float = 100.0, nt: int = 101, amp: float = 1.0, sigma: float = 1.25,
                     sigmat: float = 2.0, cs: float = 0.2, rho: float = 1.0, cfl: float = 0.5, fd: str = "SBP4",
                     forcing_file: str | None = None) -> str:
    """Mode III, one block of n x n nodes over [-L/2, L/2]^2 with absorbing
    sides, driven by the source_list 'Forcing' term (source.f90:299-312):
    DF(vz) += amp*exp(-(x/sigma)^2/2 - (y/sigma)^2/2) * exp(-((t-4 sigmat)/sigmat)^2/2) / (sigmat*sqrt(2 pi)),
    or, with `forcing_file`, by that file's frames instead."""
    h = 0.5 * L
    src = (f"forcing_from_file=T, forcing_filename='{forcing_file}'" if forcing_file else
           f"problem='Forcing', gauss_amp={_f(amp)}, gauss_sigma={_f(sigma)}, gauss_sigmat={_f(sigmat)}")
    return f"""&problem_list name='gaussian_forcing', nt={nt}, CFL={_f(cfl)} , RKorder=4 /
&domain_list mode=3, FDmethod='{fd}', nblocks_x=1, nblocks_y=1 /
!---BLOCK1---
&grid_list nx={n}, ny={n}, LB={_f(-h)},{_f(-h)}, LT={_f(-h)},{_f(h)}, RB={_f(h)},{_f(-h)}, RT={_f(h)},{_f(h)} /
&boundaries_list bcL='absorbing', bcR='absorbing', bcB='absorbing', bcT='absorbing' /
&source_list {src} /
&material_list rho={_f(rho)}, cs={_f(cs)} /
"""


def write_forcing_file(path: str | Path, x: np.ndarray, y: np.ndarray, times, nF: int, field: int, fn) -> None:
    """Forcing file (init_forcing_from_file / load_forcing, source.f90:409-502):
    for each time, nF real*8 planes over the global grid (i fastest), plane
    `field` = fn(x, y, t) and the others zero.  x, y: node coordinates, shape (ny, nx)."""
    with open(path, "wb") as f:
        for t in times:
            frame = np.zeros((nF,) + x.shape)
            frame[field] = fn(x, y, t)
            frame.astype(np.float64).tofile(f)


def rupture_sw(nx: int = 1601, ny: int = 801, h: float = 0.025, nt: int = 4001, rk: int = 4, cfl: float = 0.5,
               fd: str = "SBP4", patch_half_width: float = 1.5, cdiss: float = 0.0) -> str:
    """Mode II dynamic rupture on a planar fault y = 0 between two blocks of
    nx x ny nodes (spacing h km), linear slip-weakening friction, uniform
    prestress syy = -110 MPa, sxy = 65 MPa, and an 80 MPa nucleation patch."""
    Lx = (nx - 1) * h
    Ly = (ny - 1) * h
    x0, x1 = -0.5 * Lx, 0.5 * Lx
    blk = _operator(cdiss) + """&material_list rho=2.67d0, cs=3.464d0, cp=6d0 /
&fields_list syy0=-110d0, sxy0=65d0 /
"""
    return f"""&problem_list name='rupture_sw', nt={nt}, CFL={_f(cfl)}, RKorder={rk} /
&domain_list mode=2, FDmethod='{fd}', nblocks_x=1, nblocks_y=2 /
!---BLOCK1---
&grid_list nx={nx}, ny={ny}, LB={_f(x0)},{_f(-Ly)}, LT={_f(x0)},0d0, RB={_f(x1)},{_f(-Ly)}, RT={_f(x1)},0d0 /
&boundaries_list bcL='absorbing', bcR='absorbing', bcB='absorbing', bcT='none' /
{blk}!---BLOCK2---
&grid_list nx={nx}, ny={ny}, LB={_f(x0)},0d0, LT={_f(x0)},{_f(Ly)}, RB={_f(x1)},0d0, RT={_f(x1)},{_f(Ly)} /
&boundaries_list bcL='absorbing', bcR='absorbing', bcB='none', bcT='absorbing' /
{blk}!---IFACE1---
&interface_list coupling='friction' /
&friction_list friction_law='SW', sw%fs=0.68d0, sw%fd=0.52d0, sw%Dc=0.4d0,
  ld%shape='boxcar', ld%R={_f(patch_half_width)}, ld%S=15d0, ld%x0=0d0,
  rup_field='V', rup_threshold=1d-3 /
"""


def fractal_profile(x: np.ndarray, alpha: float, lambda_min: float, seed: int) -> tuple[np.ndarray, np.ndarray]:
    """Seeded band-limited self-similar profile y(x) (power spectral density
    proportional to k^-3, i.e. Hurst exponent 1) with rms amplitude alpha*L and
    wavelengths between lambda_min and the profile length L; returns (y, dy/dx)."""
    rng = np.random.default_rng(seed)
    n = x.size
    L = x[-1] - x[0]
    m = 4 * n
    k = np.fft.rfftfreq(m, d=(x[1] - x[0]))
    amp = np.zeros_like(k)
    band = (k >= 1.0 / L) & (k <= 1.0 / lambda_min)
    amp[band] = k[band] ** -1.5
    spec = amp * np.exp(2j * np.pi * rng.random(k.size))
    y = np.fft.irfft(spec, n=m)[:n]
    dy = np.fft.irfft(spec * 2j * np.pi * k, n=m)[:n]
    scale = alpha * L / np.sqrt(np.mean(y ** 2))
    y = y * scale
    dy = dy * scale
    y = y - y[0]  # anchor the left end at y = 0
    return y, dy


def _write(path: Path, *arrays) -> None:
    np.concatenate([np.asarray(a, dtype=np.float64).ravel() for a in arrays]).tofile(path)


def rough_fault_rs(outdir: str | Path, nx: int = 2001, ny: int = 1001, h: float = 0.02, nt: int = 6001, rk: int = 4,
                   cfl: float = 0.5, fd: str = "SBP4", seed: int = 0, alpha: float = 1e-3, Vinit: float = 1e-12,
                   tp: bool = False) -> str:
    """Mode II regularised rate-and-state (flash-heating slip law 'RFL') on a
    rough fault between two curvilinear blocks.  Writes the fault curve, the
    background-stress file and the initial-state file into outdir and returns
    the input text (file names relative to outdir)."""
    out = Path(outdir)
    out.mkdir(parents=True, exist_ok=True)
    Lx, Ly = (nx - 1) * h, (ny - 1) * h
    x = np.linspace(-0.5 * Lx, 0.5 * Lx, nx)
    y, dy = fractal_profile(x, alpha, 20 * h, seed)
    nrm = np.sqrt(1.0 + dy ** 2)
    # curve file (grid.f90:683-695): x, y, n1, n2; the stored normal points out of
    # the upper block (downwards); the lower block's T side flips it (grid.f90:453)
    _write(out / "fault.curve", x, y, dy / nrm, -1.0 / nrm)
    # depth-dependent effective normal stress capped at 120 MPa, shear at 0.4 N
    depth = x - x[0]
    N0 = np.minimum(120.0, 20.0 + 10.0 * depth)
    a, b, V0, f0, L, fw, Vw = 0.01, 0.014, 1e-6, 0.6, 0.4, 0.2, 0.1
    S0 = 0.4 * N0
    _write(out / "stress.dat", S0, N0)
    # state giving slip velocity Vinit under the background stress (strength()
    # of friction.f90:1066-1071 inverted for Psi)
    Psi = a * np.log(2.0 * V0 / Vinit * np.sinh(S0 / (a * N0)))
    _write(out / "state.dat", Psi)
    xa, xb = x[0], x[-1]
    ya, yb = y[0], y[-1]
    tp_list = "&thermpres_list n=64, p0=0d0 /\n" if tp else ""
    blk = """&material_list rho=2.67d0, cs=3.464d0, cp=6d0 /
"""
    return f"""&problem_list name='rough_fault_rs', nt={nt}, CFL={_f(cfl)}, RKorder={rk} /
&domain_list mode=2, FDmethod='{fd}', nblocks_x=1, nblocks_y=2 /
!---BLOCK1---
&grid_list nx={nx}, ny={ny}, LB={_f(xa)},{_f(-Ly)}, LT={_f(xa)},{_f(ya)}, RB={_f(xb)},{_f(-Ly)}, RT={_f(xb)},{_f(yb)},
  bndTfile='fault.curve' /
&boundaries_list bcL='absorbing', bcR='absorbing', bcB='absorbing', bcT='none' /
{blk}!---BLOCK2---
&grid_list nx={nx}, ny={ny}, LB={_f(xa)},{_f(ya)}, LT={_f(xa)},{_f(Ly)}, RB={_f(xb)},{_f(yb)}, RT={_f(xb)},{_f(Ly)},
  bndBfile='fault.curve' /
&boundaries_list bcL='absorbing', bcR='absorbing', bcB='none', bcT='absorbing' /
{blk}!---IFACE1---
&interface_list coupling='friction' /
&friction_list friction_law='RFL', rs%a={_f(a)}, rs%b={_f(b)}, rs%V0={_f(V0)}, rs%f0={_f(f0)}, rs%L={_f(L)},
  rs%fw={_f(fw)}, rs%Vw={_f(Vw)}, stress_file=T, stress_filename='stress.dat',
  state_file=T, state_filename='state.dat',
  ld%shape='gaussian', ld%R=3d0, ld%S=45d0, ld%x0={_f(x[nx // 2])},
  rup_field='V', rup_threshold=1d-3 /
{tp_list}"""


def heterogeneous_ricker(outdir: str | Path, n: int = 801, h: float = 0.02, nt: int = 2001, rk: int = 4,
                         cfl: float = 0.5, fd: str = "SBP4", seed: int = 0, std: float = 0.1, corr: float = 0.4,
                         f_peak: float = 5.0, rho_scale: float = 1.0) -> str:
    """Mode III wave in a heterogeneous block: shear modulus and density are
    seeded Gaussian random fields (relative std `std`, correlation length
    `corr` km) about 32 GPa and 2.67 g/cm^3; Ricker point force at a seeded node."""
    out = Path(outdir)
    out.mkdir(parents=True, exist_ok=True)
    rng = np.random.default_rng(seed)
    L = (n - 1) * h

    def grf(r):
        w = r.standard_normal((n, n))
        k = np.fft.fftfreq(n, d=h)
        kx, ky = np.meshgrid(k, k, indexing="ij")
        filt = np.exp(-0.5 * (2 * np.pi) ** 2 * (kx ** 2 + ky ** 2) * (corr / 2) ** 2)
        g = np.real(np.fft.ifft2(np.fft.fft2(w) * filt))
        return g / g.std()

    rho = 2.67 * rho_scale * (1.0 + std * grf(rng))
    G = 32.0 * (1.0 + std * grf(rng))
    cs = np.sqrt(G / rho)
    cp = np.sqrt(3.0) * cs
    # medium file (material.f90:278-321): rho, cs, cp over the global grid, i fastest
    _write(out / "medium.dat", rho.T, cs.T, cp.T)
    i0, j0 = rng.integers(n // 4, 3 * n // 4, size=2)
    x0, y0 = i0 * h + 0.37 * h, j0 * h + 0.61 * h
    T = 1.0 / f_peak
    return f"""&problem_list name='heterogeneous_ricker', nt={nt}, CFL={_f(cfl)}, RKorder={rk} /
&domain_list mode=3, FDmethod='{fd}', nblocks_x=1, nblocks_y=1 /
!---BLOCK1---
&grid_list nx={n}, ny={n}, LB=0d0,0d0, LT=0d0,{_f(L)}, RB={_f(L)},0d0, RT={_f(L)},{_f(L)} /
&boundaries_list bcL='absorbing', bcR='absorbing', bcB='absorbing', bcT='free' /
&material_list heterogeneous=T, filename='medium.dat', rho=2.67d0, cs=3.464d0 /
!---END---
&source_list x0={_f(x0)}, y0={_f(y0)}, Fz=1d0, source_time_function='Ricker', t_center={_f(1.2 * T)}, t_duration={_f(T)} /
"""


def heterogeneous_rs_fault(outdir: str | Path, n: int = 41, h: float = 0.25, nt: int = 41, rk: int = 4,
                           cfl: float = 0.5, fd: str = "SBP4", law: str = "RAL", seed: int = 0, std: float = 0.05,
                           corr: float = 1.0, coupling: str = "friction") -> str:
    """Mode III rupture on a rate-and-state fault y = 0 between two
    heterogeneous blocks of n x (n//2 + 1) nodes: density and shear modulus
    are seeded Gaussian random fields (relative std `std`, correlation length
    `corr` km) about 2.67 g/cm^3 and 32 GPa over the global grid, and a
    Gaussian shear load nucleates slip at the centre."""
    out = Path(outdir)
    out.mkdir(parents=True, exist_ok=True)
    rng = np.random.default_rng(seed)
    m = n // 2 + 1
    L, W = (n - 1) * h, (m - 1) * h

    def grf(shape):
        w = rng.standard_normal(shape)
        kx = np.fft.fftfreq(shape[0], d=h)[:, None]
        ky = np.fft.fftfreq(shape[1], d=h)[None, :]
        filt = np.exp(-0.5 * (2 * np.pi) ** 2 * (kx ** 2 + ky ** 2) * (corr / 2) ** 2)
        g = np.real(np.fft.ifft2(np.fft.fft2(w) * filt))
        return g / g.std()

    # global grid: block 1 rows 1..m, block 2 rows m+1..2m; arrays (nx, ny), i fastest on disk
    rho = 2.67 * (1.0 + std * grf((n, 2 * m)))
    G = 32.0 * (1.0 + std * grf((n, 2 * m)))
    cs = np.sqrt(G / rho)
    _write(out / "medium.dat", rho.T, cs.T, np.sqrt(3.0) * cs.T)
    g1 = f"nx={n}, ny={m}, LB={_f(-L / 2)},{_f(-W)}, LT={_f(-L / 2)},0d0, RB={_f(L / 2)},{_f(-W)}, RT={_f(L / 2)},0d0"
    g2 = f"nx={n}, ny={m}, LB={_f(-L / 2)},0d0, LT={_f(-L / 2)},{_f(W)}, RB={_f(L / 2)},0d0, RT={_f(L / 2)},{_f(W)}"
    mat = "&material_list heterogeneous=T, filename='medium.dat', rho=2.67d0, cs=3.464d0 /"
    fields = "&fields_list syy0=-100d0, syz0=58d0 /"
    friction = (f"&friction_list friction_law='{law}', rs%a=0.01d0, rs%b=0.014d0, rs%V0=1d-6, rs%f0=0.6d0, "
                "rs%L=0.05d0, rs%fw=0.2d0, rs%Vw=0.1d0, Psi0=0.6d0, ld%shape='gaussian', ld%R=1.5d0, "
                "ld%S=20d0, ld%x0=0d0, ld%y0=0d0, ld%T=0d0 /\n") if coupling == "friction" else ""
    return f"""&problem_list name='heterogeneous_rs_fault', nt={nt}, CFL={_f(cfl)}, RKorder={rk} /
&domain_list mode=3, FDmethod='{fd}', nblocks_x=1, nblocks_y=2 /
!---BLOCK1---
&grid_list {g1} /
&boundaries_list bcL='absorbing', bcR='absorbing', bcB='absorbing', bcT='none' /
{mat}
{fields}
!---BLOCK2---
&grid_list {g2} /
&boundaries_list bcL='absorbing', bcR='absorbing', bcB='none', bcT='free' /
{mat}
{fields}
!---IFACE1---
&interface_list coupling='{coupling}', direction='y' /
{friction}"""


def von_karman_1d(n: int, h: float, hurst: float, corr: float, seed: int) -> np.ndarray:
    """Seeded 1-D von Karman random field on n points of spacing h: power
    spectral density proportional to (1 + (k a)^2)^-(H + 1/2) with k the
    angular wavenumber and a the correlation length; zero mean, unit std."""
    rng = np.random.default_rng(seed)
    m = 2 * n
    k = 2.0 * np.pi * np.fft.rfftfreq(m, d=h)
    psd = (1.0 + (k * corr) ** 2) ** (-(hurst + 0.5))
    w = np.fft.rfft(rng.standard_normal(m)) * np.sqrt(psd)
    w[0] = 0.0
    f = np.fft.irfft(w, n=m)[:n]
    f = f - f.mean()
    return f / f.std()


ENSEMBLE_GRIDS = ((401, 401), (801, 401), (801, 801), (1601, 801))


def ensemble_grid(seed: int) -> tuple[int, int]:
    """Per-block grid of ensemble instance `seed`: a seeded uniform draw from
    401x401, 801x401, 801x801 and 1601x801 (nx x ny)."""
    return ENSEMBLE_GRIDS[int(np.random.default_rng(1000 + seed).integers(len(ENSEMBLE_GRIDS)))]


def ensemble_instance(outdir: str | Path, seed: int, nx: int | None = None, ny: int | None = None,
                      h: float = 0.025, nt: int = 1001, rk: int = 4, cfl: float = 0.5, fd: str = "SBP4",
                      N0: float = 120.0, Vinit: float = 1e-12, hurst: float = 0.8, corr: float = 2.0,
                      std: float = 0.1, strength_frac: float = 0.6) -> str:
    """One instance of the rupture ensemble: mode II regularised rate-and-state
    (slip law with flash heating, 'RFL', the rough-fault friction parameters)
    on a planar fault y = 0 between two blocks of nx x ny nodes (spacing h km).
    Initial shear stress S0 = strength_frac * f0 * N0 * (1 + std * z) with z a
    seeded von Karman field (Hurst `hurst`, correlation length `corr` km);
    the state gives slip velocity Vinit under it; a Gaussian overstress at
    the fault centre nucleates rupture.  Writes stress and state files into
    outdir and returns the input text (file names relative to outdir)."""
    out = Path(outdir)
    out.mkdir(parents=True, exist_ok=True)
    if nx is None or ny is None:
        nx, ny = ensemble_grid(seed)
    Lx, Ly = (nx - 1) * h, (ny - 1) * h
    a, b, V0, f0, L, fw, Vw = 0.01, 0.014, 1e-6, 0.6, 0.4, 0.2, 0.1
    z = von_karman_1d(nx, h, hurst, corr, seed)
    N0a = np.full(nx, N0)
    S0 = strength_frac * f0 * N0a * (1.0 + std * z)
    _write(out / f"stress_{seed}.dat", S0, N0a)
    Psi = a * np.log(2.0 * V0 / Vinit * np.sinh(S0 / (a * N0a)))
    _write(out / f"state_{seed}.dat", Psi)
    x0, x1 = -0.5 * Lx, 0.5 * Lx
    blk = """&material_list rho=2.67d0, cs=3.464d0, cp=6d0 /
"""
    return f"""&problem_list name='ensemble_{seed}', nt={nt}, CFL={_f(cfl)}, RKorder={rk} /
&domain_list mode=2, FDmethod='{fd}', nblocks_x=1, nblocks_y=2 /
!---BLOCK1---
&grid_list nx={nx}, ny={ny}, LB={_f(x0)},{_f(-Ly)}, LT={_f(x0)},0d0, RB={_f(x1)},{_f(-Ly)}, RT={_f(x1)},0d0 /
&boundaries_list bcL='absorbing', bcR='absorbing', bcB='absorbing', bcT='none' /
{blk}!---BLOCK2---
&grid_list nx={nx}, ny={ny}, LB={_f(x0)},0d0, LT={_f(x0)},{_f(Ly)}, RB={_f(x1)},0d0, RT={_f(x1)},{_f(Ly)} /
&boundaries_list bcL='absorbing', bcR='absorbing', bcB='none', bcT='absorbing' /
{blk}!---IFACE1---
&interface_list coupling='friction' /
&friction_list friction_law='RFL', rs%a={_f(a)}, rs%b={_f(b)}, rs%V0={_f(V0)}, rs%f0={_f(f0)}, rs%L={_f(L)},
  rs%fw={_f(fw)}, rs%Vw={_f(Vw)}, stress_file=T, stress_filename='stress_{seed}.dat',
  state_file=T, state_filename='state_{seed}.dat',
  ld%shape='gaussian', ld%R=3d0, ld%S=45d0, ld%x0=0d0,
  rup_field='V', rup_threshold=1d-3 /
"""
