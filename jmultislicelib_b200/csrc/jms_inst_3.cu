// jms_inst_3.cu -- pass instantiations for plans P480, P512a.
#include "jms_passes.cuh"
#include "jms_sizes.h"

namespace jms {
JMS_INSTANTIATE(P480)
JMS_INSTANTIATE(P512a)
} // namespace jms
