// cluster_kernels.cu -- kernel family CLUSTER (volumes larger than one SM's shared memory).
#include "internal.h"

namespace fft3d {

void register_cluster_kernels(std::vector<KernelEntry> &out) { (void)out; }

}  // namespace fft3d
