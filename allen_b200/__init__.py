"""B200-native VELO super-pixel reconstruction (Allen veloSP chain)."""
