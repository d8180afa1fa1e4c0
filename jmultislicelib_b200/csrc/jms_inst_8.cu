// jms_inst_8.cu -- pass instantiations for plans P2048a, P2048b.
#include "jms_passes.cuh"
#include "jms_sizes.h"

namespace jms {
JMS_INSTANTIATE(P2048a)
JMS_INSTANTIATE(P2048b)
} // namespace jms
