// jms_inst_1.cu -- pass instantiations for plans P120, P128a, P128b, P160, P180, P192, P240.
#include "jms_passes.cuh"
#include "jms_sizes.h"

namespace jms {
JMS_INSTANTIATE(P120)
JMS_INSTANTIATE(P128a)
JMS_INSTANTIATE(P128b)
JMS_INSTANTIATE(P160)
JMS_INSTANTIATE(P180)
JMS_INSTANTIATE(P192)
JMS_INSTANTIATE(P240)
} // namespace jms
