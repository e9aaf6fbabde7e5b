// Minimal stand-in for the CUDA-samples helper_string.h, which the reference's
// helper_cuda.h includes (3DGPUwithPML_1DArraySingleGPU_optimization/helper_cuda.h:41)
// but does not ship.  helper_cuda.h only calls these two functions, from
// findCudaDevice() (helper_cuda.h:779-780), which the reference never calls.
// Used only to compile the reference program as an oracle pin (oracle/Makefile).
#ifndef SGFD_REF_STUB_HELPER_STRING_H
#define SGFD_REF_STUB_HELPER_STRING_H
inline bool checkCmdLineFlag(int, const char **, const char *) { return false; }
inline int getCmdLineArgumentInt(int, const char **, const char *) { return 0; }
#endif
