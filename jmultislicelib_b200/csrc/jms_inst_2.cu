// jms_inst_2.cu -- pass instantiations for line lengths 256, 320, 384.
#include "jms_passes.cuh"

namespace jms {
JMS_INSTANTIATE(16, 16)
JMS_INSTANTIATE(16, 20)
JMS_INSTANTIATE(16, 24)
} // namespace jms
