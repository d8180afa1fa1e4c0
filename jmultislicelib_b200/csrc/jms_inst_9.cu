// jms_inst_9.cu -- pass instantiations for plan P512c.
#include "jms_passes.cuh"
#include "jms_sizes.h"

namespace jms {
JMS_INSTANTIATE(P512c)
} // namespace jms
