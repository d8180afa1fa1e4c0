// jms_inst_6.cu -- pass instantiations for line lengths 1024.
#include "jms_passes.cuh"

namespace jms {
JMS_INSTANTIATE(32, 32)
} // namespace jms
