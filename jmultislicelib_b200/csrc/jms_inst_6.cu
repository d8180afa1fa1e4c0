// jms_inst_6.cu -- pass instantiations for plans P768, P960.
#include "jms_passes.cuh"
#include "jms_sizes.h"

namespace jms {
JMS_INSTANTIATE(P768)
JMS_INSTANTIATE(P960)
} // namespace jms
