// conv_f16.cu — engine kernels and launchers for f16 image storage.
#include "conv_launch.cuh"

SRK_INSTANTIATE_CONV(__half)
