// float-precision hopping kernels, epilogue 2 (split so the instantiations compile in parallel)
#include "hop_launch.cuh"

namespace hrgpu {
template int launch_ep<float, 2>(HopArgs<float> &);
}
