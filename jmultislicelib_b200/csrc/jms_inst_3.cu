// jms_inst_3.cu -- pass instantiations for line lengths 480, 512.
#include "jms_passes.cuh"

namespace jms {
JMS_INSTANTIATE(20, 24)
JMS_INSTANTIATE(16, 32)
} // namespace jms
