// double-precision instantiation of the hopping kernels
#include "hop_launch.cuh"

namespace hrgpu {
template int launch_hop<double>(int, HopArgs<double> &);
}
