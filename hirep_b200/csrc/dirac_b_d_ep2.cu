// multi-field hopping kernels, double, epilogue 2 (split so the instantiations compile in parallel)
#include "hop_batch_launch.cuh"

namespace hrgpu {
template int launch_batch<double, 2>(TileArgs<double> &);
}
