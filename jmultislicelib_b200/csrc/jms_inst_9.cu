// jms_inst_9.cu -- pass instantiations for plans P256p, P512p (pipelined).
#include "jms_passes.cuh"
#include "jms_sizes.h"

namespace jms {
JMS_INSTANTIATE(P256p)
JMS_INSTANTIATE(P512p)
} // namespace jms
