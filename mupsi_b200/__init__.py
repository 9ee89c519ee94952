"""B200-native GPIS path-tracing hot path (mupsi): CUDA kernels behind a C ABI."""
