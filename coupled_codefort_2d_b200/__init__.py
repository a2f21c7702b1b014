"""B200-native FUGU-2D coupled-step hot path (package placeholder; filled below)."""
