"""B200 render path for MobileRT (MobileRayTracer): CUDA kernels behind the C ABI of
include/mrt_cuda.h, with Python bindings for tests and benchmarks."""
