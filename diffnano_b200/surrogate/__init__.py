"""Learned surrogate of the FDTD design loop: a Fourier neural operator whose
training and inference run on the project's BF16 tensor-core GEMM."""
