"""spiffe_b200: B200-native per-timestep PIC loop of spiffe (r-z EM PIC)."""
