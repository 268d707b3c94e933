"""cleo_b200 — B200-native super-droplet microphysics hot path with CLEO's SDM interface.

The compute path is hand-written CUDA for sm_100a in ``libcleo_b200.so`` (sources in
``cleo_b200/csrc``), reached through the C ABI of ``include/cleo_b200.h``. This package holds the
host side: the ctypes binding (:mod:`cleo_b200.abi`), parameter and grid construction mirroring
the reference factories (:mod:`cleo_b200.config`), the SDMMethods-shaped driver
(:mod:`cleo_b200.sdm`) and seeded synthetic workloads (:mod:`cleo_b200.workloads`).
"""
from . import abi, config  # noqa: F401

__all__ = ["abi", "config"]
