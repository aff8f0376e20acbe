"""pyugks_b200: B200-native UGKS time step (placeholder init, filled in below)."""
