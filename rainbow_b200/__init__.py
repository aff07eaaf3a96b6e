"""B200-native implementation of RAINBOW's prox_rigid_bodies time step (sm_100a CUDA behind a C ABI)."""
__version__ = "0.1.0"
