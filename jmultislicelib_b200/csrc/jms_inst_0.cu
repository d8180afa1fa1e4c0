// jms_inst_0.cu -- pass instantiations for line lengths 16, 24, 32, 40, 48, 64, 80, 96.
#include "jms_passes.cuh"

namespace jms {
JMS_INSTANTIATE(4, 4)
JMS_INSTANTIATE(4, 6)
JMS_INSTANTIATE(4, 8)
JMS_INSTANTIATE(5, 8)
JMS_INSTANTIATE(6, 8)
JMS_INSTANTIATE(8, 8)
JMS_INSTANTIATE(8, 10)
JMS_INSTANTIATE(8, 12)
} // namespace jms
