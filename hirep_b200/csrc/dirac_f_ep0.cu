// float-precision hopping kernels, epilogue 0 (split so the instantiations compile in parallel)
#include "hop_launch.cuh"

namespace hrgpu {
template int launch_ep<float, 0>(HopArgs<float> &);
}
