"""TEST INFRASTRUCTURE ONLY: the oracle.

Two CPU implementations of the reference's restarted-PDHG path, loaded with ctypes:

* ``liboracle_pdhg.so`` -- our plain-C FP64 restatement (oracle/pdhg_oracle.c), built by
  ``make -C oracle oracle``; it travels with the repository.
* ``libsankhya_ref.so`` -- the reference's own sources compiled in place with our harness
  (oracle/ref_harness.cpp), built by ``make -C oracle ref`` where the reference tree exists.

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may import
this package, and only as the checker or the timed CPU baseline -- never as the product.
"""
from .loader import (  # noqa: F401
    OracleResult,
    oracle_available,
    oracle_csc_multiply,
    oracle_csc_transpose_multiply,
    oracle_evaluate,
    oracle_primal_step,
    oracle_scaling,
    oracle_solve,
    oracle_spectral_norm,
    oracle_uniform_draws,
    ref_available,
    ref_farkas_check,
    ref_kkt_instance,
    ref_polish_ipm,
    ref_qp_solve,
    ref_ray_check,
    ref_read_model,
    ref_recompute_quality,
    ref_scaling,
    ref_solve,
    ref_spectral_norm,
    ref_validate,
)
from .quality import recompute_quality  # noqa: F401,E402
