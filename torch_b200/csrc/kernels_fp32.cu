// FP32 performance-form kernels (filled in below the FP64 parity form).
#include "trg_device.cuh"
#include "trg_kernels.h"
