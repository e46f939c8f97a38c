// conv_bf16.cu — engine kernels and launchers for bf16 image storage.
#include "conv_launch.cuh"

SRK_INSTANTIATE_CONV(__nv_bfloat16)
