// jms_inst_7.cu -- pass instantiations for plans P1024a, P1024b.
#include "jms_passes.cuh"
#include "jms_sizes.h"

namespace jms {
JMS_INSTANTIATE(P1024a)
JMS_INSTANTIATE(P1024b)
} // namespace jms
