"""wadi2d_b200: the uniform-grid shallow-water step of Wadi2D, B200-native (sm_100a CUDA behind a C-ABI)."""

__version__ = "0.1.0"
