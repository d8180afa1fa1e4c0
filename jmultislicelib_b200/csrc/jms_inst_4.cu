// jms_inst_4.cu -- pass instantiations for line lengths 640, 720.
#include "jms_passes.cuh"

namespace jms {
JMS_INSTANTIATE(20, 32)
JMS_INSTANTIATE(24, 30)
} // namespace jms
