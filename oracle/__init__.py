"""CPU oracle for the vkzg hot path -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this
package, and only as the checker.  See vkzg_oracle.h for what it restates.
"""
from .oracle import Oracle, OracleTables, build  # noqa: F401
