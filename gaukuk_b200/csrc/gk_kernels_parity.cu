// Kernels in parity mode: compiled with -fmad=false, IEEE division and square
// root, every HLLC side evaluated as the reference does (hllc.cpp:71-94).
#define GK_NS gk_parity
#define GK_SEL 0
#define GK_FASTMATH 0
#include "gk_kernels.cuh"

