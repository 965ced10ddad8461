// FP64 build compiled with -fmad=false: every multiply and add rounds
// separately, as in the reference's x86-64 build, so the step reproduces the
// reference operation for operation (the parity build).
#define IBGPU_KNS exact
#include "kernels.cuh"
#include "amr_kernels.cuh"
#include "launchers.h"
