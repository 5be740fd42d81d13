// Kernels in fast mode: FMA contraction allowed, only the selected HLLC side
// evaluated.
#define GK_NS gk_fast
#define GK_SEL true
#include "gk_kernels.cuh"
