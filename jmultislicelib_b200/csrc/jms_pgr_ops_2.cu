// jms_pgr_ops_2.cu -- phase-grating generator transforms, length group 2.
#include "jms_pgr_t.cuh"

namespace jms {
const PgrOps* pgr_ops_2(int n)
{
	static const PgrOps ops[] = {JMS_DEFAULT_PLANS_2(JMS_PGR_OPS)};
	for (const PgrOps& o : ops)
		if (o.n == n) return &o;
	return nullptr;
}
} // namespace jms
