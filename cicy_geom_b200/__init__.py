"""B200-native (sm_100a) network-to-conductance hot path of CICY_geom.

The product is the shared library libcicy_b200.so (CUDA kernels + C ABI,
include/cicy_b200.h); this package holds its build script and a thin ctypes
host layer that mirrors the upstream class interfaces.
"""
from .network import HostNetwork, NetworkConfig, generate_cnt_network, write_read_network_files  # noqa: F401
