"""CPU oracle of the bonded-particle DEM step and the harness around the
reference's own kernels.  Test infrastructure only: imported by tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg, never by the product."""
