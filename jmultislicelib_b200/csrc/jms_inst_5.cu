// jms_inst_5.cu -- pass instantiations for plans P640, P720.
#include "jms_passes.cuh"
#include "jms_sizes.h"

namespace jms {
JMS_INSTANTIATE(P640)
JMS_INSTANTIATE(P720)
} // namespace jms
