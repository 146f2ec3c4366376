// Device bandwidth measurement for roofline reporting.
#pragma once
#include <cuda_runtime.h>

namespace nnk {

// L2 read bandwidth (GB/s) of the current device: the best of a streaming
// read of a 24 and a 48 MiB buffer (held in L2 after a warm-up pass) by 8
// and 16 blocks of 256 threads per SM, timed with events on st.
double measure_l2_read_gbs(cudaStream_t st);

}  // namespace nnk
