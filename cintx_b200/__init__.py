"""B200 two-electron Gaussian integrals with libcint's calling conventions.

The compute path is libcintx_cuda.so (csrc/, built by build.py for sm_100a).  This module is
the Python host mirror of the libcint-style interface that callers such as PySCF drivers use
through ctypes:

    int2e_sph(shls, atm, bas, env, opt=None, dims=None) -> (block, nonzero)
    int2e_cart / int3c2e_sph / int3c2e_cart / int2c2e_sph / int2c2e_cart
    Optimizer(atm, bas, env, family)        # int2e_optimizer / CINTdel_optimizer
    Plan.shells(opt, family, tuples, sph)   # batched device evaluation
    Plan.screened(opt, cutoff, sph, chunk)  # all unique Schwarz-surviving int2e quartets

There is no CPU fallback: the first use of any of these names loads the shared object and
raises ImportError when it is missing; every compute call needs a CUDA device.  The
synthetic-molecule builders in `molecules` are plain Python and load nothing.
"""
from __future__ import annotations

INT2E, INT3C2E, INT2C2E = 0, 1, 2

_API = {"CintxError", "Optimizer", "Plan", "int2c2e_cart", "int2c2e_sph", "int2e_cart", "int2e_sph",
        "int3c2e_cart", "int3c2e_sph", "lib", "launch_count", "rys_roots", "rys_t2_batch", "last_error",
        "RysNet", "ao_loc", "int2e_ip1_sph", "int2e_ip1_cart", "int3c2e_ip1_sph", "int3c2e_ip1_cart",
        "ip1_eval", "ip1_len", "tuned_shapes", "load_tuned_shapes"}


def __getattr__(name):
    if name in _API:
        from . import _lib
        return getattr(_lib, name)
    raise AttributeError(name)
