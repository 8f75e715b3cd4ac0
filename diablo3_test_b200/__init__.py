"""libdiablo_gpu: DIABLO 3's RK3/Crank-Nicolson channel step on one B200.

The product is the CUDA library ``libdiablo_gpu.so`` behind the C ABI in
``include/diablo_gpu.h``; this package holds its sources (``csrc/``), the
in-tree build (``build.py``), the ctypes binding (``_lib.py``), the Python
front end (``channel.Channel``), run parameters (``config``), grids
(``grid``) and initial conditions (``ics``).
"""
from .config import ChannelParams, FP64, MIXED, read_input_toml  # noqa: F401
