"""CPU oracle and CPU port of the nonbonded + PME path: test and baseline
infrastructure only (tests/, __graft_entry__.smoke() and bench.py's CPU
baseline leg import it, as the checker; the product never does)."""
