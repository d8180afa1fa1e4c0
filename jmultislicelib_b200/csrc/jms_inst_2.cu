// jms_inst_2.cu -- pass instantiations for plans P256a, P256b, P320, P384.
#include "jms_passes.cuh"
#include "jms_sizes.h"

namespace jms {
JMS_INSTANTIATE(P256a)
JMS_INSTANTIATE(P256b)
JMS_INSTANTIATE(P320)
JMS_INSTANTIATE(P384)
} // namespace jms
