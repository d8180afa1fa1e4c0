// jms_inst_0.cu -- pass instantiations for plans P16, P24, P32, P40, P48, P64a, P64b, P80, P96.
#include "jms_passes.cuh"
#include "jms_sizes.h"

namespace jms {
JMS_INSTANTIATE(P16)
JMS_INSTANTIATE(P24)
JMS_INSTANTIATE(P32)
JMS_INSTANTIATE(P40)
JMS_INSTANTIATE(P48)
JMS_INSTANTIATE(P64a)
JMS_INSTANTIATE(P64b)
JMS_INSTANTIATE(P80)
JMS_INSTANTIATE(P96)
} // namespace jms
