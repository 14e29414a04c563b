// kernels_mixed.cu -- mixed-precision kernels (FP64 trajectory and retarded phase, FP32 amplitudes).
#include "kernels.h"
