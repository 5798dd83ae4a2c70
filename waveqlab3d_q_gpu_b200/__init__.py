"""B200-native WaveQLab3D per-step volume update (sm_100a CUDA behind a C ABI)."""
