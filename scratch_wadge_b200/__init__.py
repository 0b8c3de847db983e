"""scratch_wadge_b200 — B200-native entropy-stable flux-differencing RHS."""
