// multi-field hopping kernels, double, epilogue 1 (split so the instantiations compile in parallel)
#include "hop_batch_launch.cuh"

namespace hrgpu {
template int launch_batch<double, 1>(TileArgs<double> &);
}
