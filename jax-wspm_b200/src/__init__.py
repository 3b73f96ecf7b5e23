"""Drop-in mirror of the reference's ``src`` package (JAX-WSPM) on B200 CUDA kernels."""
