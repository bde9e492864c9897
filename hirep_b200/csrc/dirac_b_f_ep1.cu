// multi-field hopping kernels, float, epilogue 1 (split so the instantiations compile in parallel)
#include "hop_batch_launch.cuh"

namespace hrgpu {
template int launch_batch<float, 1>(TileArgs<float> &);
}
