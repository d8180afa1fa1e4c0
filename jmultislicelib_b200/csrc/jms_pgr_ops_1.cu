// jms_pgr_ops_1.cu -- phase-grating generator transforms, length group 1.
#include "jms_pgr_t.cuh"

namespace jms {
const PgrOps* pgr_ops_1(int n)
{
	static const PgrOps ops[] = {JMS_DEFAULT_PLANS_1(JMS_PGR_OPS)};
	for (const PgrOps& o : ops)
		if (o.n == n) return &o;
	return nullptr;
}
} // namespace jms
