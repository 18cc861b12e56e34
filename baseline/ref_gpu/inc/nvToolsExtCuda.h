// Stand-in for the CUDA 10 header that cuda_utils.cu:6 includes; NVTX 3 provides the calls.
#pragma once
#include <nvtx3/nvToolsExt.h>
