// jms_inst_5.cu -- pass instantiations for line lengths 768, 960.
#include "jms_passes.cuh"

namespace jms {
JMS_INSTANTIATE(24, 32)
JMS_INSTANTIATE(30, 32)
} // namespace jms
