// jms_inst_4.cu -- pass instantiations for plan P512b.
#include "jms_passes.cuh"
#include "jms_sizes.h"

namespace jms {
JMS_INSTANTIATE(P512b)
} // namespace jms
