// jms_launch.cuh -- sizing of persistent grids.
#pragma once
#include <cuda_runtime.h>

namespace jms {

// CTAs of kern (threads per CTA, dynamic shared memory smem) that fit on one
// SM at once, from its registers and shared memory (after selecting the
// largest shared-memory carveout for it); at least 1, at most cap.
template <class K>
cudaError_t resident_ctas(K kern, int threads, int smem, int cap, int* per_sm)
{
	cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
	if (e != cudaSuccess) return e;
	int dev = 0, regs_sm = 0, smem_sm = 0, smem_res = 0;
	cudaGetDevice(&dev);
	cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev);
	cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
	cudaDeviceGetAttribute(&smem_res, cudaDevAttrReservedSharedMemoryPerBlock, dev);
	cudaFuncAttributes fa;
	e = cudaFuncGetAttributes(&fa, kern);
	if (e != cudaSuccess) return e;
	const int warps = (threads + 31) / 32;
	const int regs_cta = ((fa.numRegs * 32 + 255) / 256) * 256 * warps;   // per-warp allocation granularity 256
	const int by_regs = regs_sm / (regs_cta > 0 ? regs_cta : 1);
	const int by_smem = smem_sm / (smem + (int)fa.sharedSizeBytes + smem_res);
	const int by_warps = 64 / (warps > 0 ? warps : 1);
	int n = by_regs < by_smem ? by_regs : by_smem;
	n = n < by_warps ? n : by_warps;
	n = n < cap ? n : cap;
	*per_sm = n < 1 ? 1 : n;
	return cudaSuccess;
}

} // namespace jms
