"""FP64 CPU oracle — TEST INFRASTRUCTURE ONLY.

Imported by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as
the checker.  The product (multigridsoftbody_b200, libmgsb.so) never imports it.
"""
from .binding import Oracle, build_oracle, ORACLE_LIB  # noqa: F401
