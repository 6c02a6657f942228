"""CPU oracle (checker) for the sharded additive-FFT Reed-Solomon path.

Test infrastructure only: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline / reference legs of bench.py.  The product never imports it.
"""
