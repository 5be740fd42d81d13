// Kernels in parity mode: compiled with -fmad=false, every HLLC side
// evaluated as the reference does (hllc.cpp:71-94).
#define GK_NS gk_parity
#define GK_SEL false
#include "gk_kernels.cuh"
