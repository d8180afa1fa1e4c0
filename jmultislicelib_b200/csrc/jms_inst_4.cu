// jms_inst_4.cu -- pass instantiations for plans P512b, P512c.
#include "jms_passes.cuh"
#include "jms_sizes.h"

namespace jms {
JMS_INSTANTIATE(P512b)
JMS_INSTANTIATE(P512c)
} // namespace jms
