"""CPU oracle for the per-placement field solve. TEST INFRASTRUCTURE ONLY.

Loaded by the tests, the smoke check and the benchmark's CPU-baseline arm to check and time
against; never by the cunibs_b200 product path. See oracle.cpp for the restated algorithm.
"""

from .binding import Oracle, OracleParams, build_oracle, oracle_dadt, oracle_l1_dinv_f32, oracle_select_size4, oracle_summary, oracle_weighted_quantiles  # noqa: F401
