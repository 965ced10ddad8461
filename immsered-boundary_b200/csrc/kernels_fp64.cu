// FP64 (contracted multiply-adds) and mixed-precision builds of the step kernels.
#define IBGPU_KNS fast
#include "kernels.cuh"
#include "launchers.h"
