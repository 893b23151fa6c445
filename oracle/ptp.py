"""CPU ORACLE — test infrastructure. PTP table shared with the host code.

The table itself is pinned against the reference dict (fml/arad.py:43-68)
by tests/test_oracle_pins.py through tests/golden/reference_tables.json.
"""
from fml_b200.data import PTP, NUCLEAR_CHARGE, ptp_of  # noqa: F401
