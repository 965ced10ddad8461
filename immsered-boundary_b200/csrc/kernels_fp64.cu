// FP64 (contracted multiply-adds) and mixed-precision builds of the step kernels.
#define IBGPU_KNS fast
#define IBGPU_FAST_BUILD 1
#include "kernels.cuh"
#include "amr_kernels.cuh"
#include "launchers.h"
