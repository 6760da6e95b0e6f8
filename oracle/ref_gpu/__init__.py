"""Reference kernels.cu on the GPU: build recipe and replay (test and baseline infrastructure)."""
