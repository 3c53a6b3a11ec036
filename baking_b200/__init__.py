"""B200-native MLS-MPM baking substep (sm_100a CUDA kernels behind a C-ABI)."""
