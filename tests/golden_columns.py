"""Column lists of the diagnostics fixture (tests/golden/make_golden.py)."""
SNAP_COLUMNS = ["z", "r", "pz", "pr", "pphi", "q", "r0", "z0", "t0", "generation", "particleID", "status"]
FLD_COLUMNS = ["z", "r", "rho", "Ez", "Er", "Bphi", "Jz", "Jr", "EzImposed", "ErImposed"]

# add_on_axis_fields' fields_used table (onAxisFields.c:130-170)
ONAXIS_COLUMNS = ["z", "Ez", "Er/r", "Bphi/r"]

# integrate's status file (setUpStatusOutputFile, status_pr.c:454-499)
STATUS_COLUMNS = ["t", "JCathode", "KineticEnergy", "FieldEnergy", "TotalEnergy", "Charge", "EzAbsMax", "ErAbsMax",
                  "Particles", "NewParticles", "SecondaryParticles", "zMax", "zMin", "zAve", "zRMS", "zStDev",
                  "rMax", "rMin", "rAve", "rRMS", "rStDev", "pzMax", "pzMin", "pzAve", "pzRMS", "pzStDev", "prMax",
                  "prMin", "prAve", "prRMS", "prStDev", "EzOOEMin", "EzOOEMax"]
