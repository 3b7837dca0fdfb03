"""B200-native engine for FDMAP's explicit time step (SBP-SAT elastodynamics with
frictional faults), behind a C ABI that FDMAP's Fortran driver can call.

Public Python surface (a mirror of the reference's host interface):
  init_domain, HostDomain, GpuDomain  -- fdmap_github_b200.domain
  GpuEnsemble                         -- batched independent instances
  GpuAdjoint                          -- misfit gradient (forward/backward pair)
  FdmapError                          -- raised on any non-zero status
"""
from .domain import GpuAdjoint, GpuDomain, GpuEnsemble, HostDomain, init_domain, init_domains  # noqa: F401
from .native import FAULT_FIELDS, FdmapError  # noqa: F401

__all__ = ["init_domain", "init_domains", "HostDomain", "GpuDomain", "GpuEnsemble", "GpuAdjoint", "FdmapError", "FAULT_FIELDS"]
