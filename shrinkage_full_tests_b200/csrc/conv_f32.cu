// conv_f32.cu — engine kernels and launchers for f32 image storage.
#include "conv_launch.cuh"

SRK_INSTANTIATE_CONV(float)
