"""Column lists of the diagnostics fixture (tests/golden/make_golden.py)."""
SNAP_COLUMNS = ["z", "r", "pz", "pr", "pphi", "q", "r0", "z0", "t0", "generation", "particleID", "status"]
FLD_COLUMNS = ["z", "r", "rho", "Ez", "Er", "Bphi", "Jz", "Jr", "EzImposed", "ErImposed"]
