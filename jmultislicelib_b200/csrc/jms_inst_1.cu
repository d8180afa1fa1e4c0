// jms_inst_1.cu -- pass instantiations for line lengths 120, 128, 160, 192, 240.
#include "jms_passes.cuh"

namespace jms {
JMS_INSTANTIATE(10, 12)
JMS_INSTANTIATE(8, 16)
JMS_INSTANTIATE(10, 16)
JMS_INSTANTIATE(12, 16)
JMS_INSTANTIATE(15, 16)
} // namespace jms
