"""CPU oracle of the filtered group-by (test infrastructure only: the parity
checker of tests/ and smoke(), and bench.py's CPU baseline)."""
