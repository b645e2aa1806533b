"""winds-master_b200: sm_100a engine for WInDS's induced-velocity hot path.

The compute lives in ``libwinds_bs.so`` (CUDA kernels + C ABI, built in-tree
by ``build.py``); this package is the Python host side of that boundary:

* :func:`BiotSavart` mirrors ``[uind, L] = BiotSavart(F1,F2,P,gamma,rc,d,co,type)``
  (``core/BiotSavart.m:1``) on host arrays;
* :func:`BiotSavartMex` mirrors the 11-argument MEX call
  (``cuda/source/BiotSavartMex.cu:688``) through the library's own
  ``mexFunction``;
* :func:`eval_device` evaluates device-resident (torch) arrays without copies.

There is no CPU fallback: every entry point raises when the library is not
built or no CUDA device is present.

The directory name contains a hyphen; import it with
``importlib.import_module("winds-master_b200")``.
"""
from __future__ import annotations

from .bs import (  # noqa: F401
    LIB_PATH,
    WindsError,
    BiotSavart,
    BiotSavartMex,
    eval_device,
    eval_host,
    last_stats,
    last_core_free,
    last_chained,
    lib,
    set_tuning,
    set_layout,
    get_tuning,
    set_autotune,
    sync,
)
