// jms_pgr_t.cuh -- line-transform kernels of the phase-grating generator
// (templates on the line plan); instantiated per length group in
// jms_pgr_ops_*.cu.
#pragma once
#include "jms_passes.cuh"
#include "jms_pgr.h"
#include "jms_sizes.h"

namespace jms {

// Rows: IFT_x in place, natural order in and out.
template <class PL>
__global__ void __launch_bounds__(row_lines<PL>() * PL::TMAX)
k_pgr_rows_inv(float2* work, long long gstride, int ny, const float2* tw)
{
	constexpr int N = PL::N, L = row_lines<PL>();
	using T = RowTileOf<PL>;
	extern __shared__ float2 sm[];
	const int tid = threadIdx.x, g = blockIdx.y, row0 = blockIdx.x * L;
	const int nval = min(L, ny - row0);
	float2* W = work + (long long)g * gstride;
	float2 v[PL::RM];
	#pragma unroll
	for (int m = 0; m < PL::RM; m++) v[m] = make_float2(0.f, 0.f);
	int line, j;
	T::template role<PL::T>(tid, line, j);
	if (line < nval && j < PL::T) {
		const float2* src = W + (long long)(row0 + line) * N;
		#pragma unroll
		for (int m = 0; m < PL::A; m++) v[m] = src[j + PL::B * m];
	}
	PL::template to_mid<true, T>(v, sm, TwGlobal{tw}, tid);
	int pos;
	T::template role<PL::TMID>(tid, line, pos);
	if (line < nval && pos < PL::TMID) {
		float2* dst = W + (long long)(row0 + line) * N;
		#pragma unroll
		for (int e = 0; e < PL::EMID; e++) dst[PL::mid(pos, e)] = v[e];
	}
}

// t = exp(i c V'): the phase c Re V' is formed and reduced in FP64
__device__ __forceinline__ float2 pot_to_pgr(float2 v, double c)
{
	double t = c * (double)v.x * 0.15915494309189535;   // turns
	t -= floor(t);
	float s, co;
	sincospif(2.f * (float)t, &s, &co);
	const float amp = expf(-(float)(c * (double)v.y));
	return make_float2(amp * co, amp * s);
}

// Columns: IFT_y -> [exp(i c V')] -> [FT_y]; src may equal dst.
template <class PL, int MODE>
__global__ void __launch_bounds__(PL::CC * PL::TMAX)
k_pgr_cols(const float2* src, float2* dst, long long gstride, int nx, double c, const float2* tw)
{
	constexpr int C = PL::CC;
	using T = ColTile<C>;
	extern __shared__ float2 sm[];
	const int tid = threadIdx.x, g = blockIdx.y, col0 = blockIdx.x * C;
	const int nval = min(C, nx - col0);
	const float2* S = src + (long long)g * gstride + col0;
	float2* D = dst + (long long)g * gstride + col0;
	float2 v[PL::RM];
	#pragma unroll
	for (int m = 0; m < PL::RM; m++) v[m] = make_float2(0.f, 0.f);
	int cc, j;
	T::template role<PL::T>(tid, cc, j);
	if (cc < nval && j < PL::T) {
		#pragma unroll
		for (int m = 0; m < PL::A; m++) v[m] = S[(long long)(j + PL::B * m) * nx + cc];
	}
	PL::template to_mid<true, T>(v, sm, TwGlobal{tw}, tid);
	int pos;
	T::template role<PL::TMID>(tid, cc, pos);
	const bool act = cc < nval && pos < PL::TMID;
	if (MODE != kPgrColInv && act) {
		#pragma unroll
		for (int e = 0; e < PL::EMID; e++) v[e] = pot_to_pgr(v[e], c);
	}
	if constexpr (MODE == kPgrColExpFt) {
		PL::template from_mid<false, T>(v, sm, TwGlobal{tw}, tid);
		T::template role<PL::T>(tid, cc, j);
		if (cc < nval && j < PL::T) {
			#pragma unroll
			for (int m = 0; m < PL::A; m++) D[(long long)(j + PL::B * m) * nx + cc] = v[m];
		}
	}
	else if (act) {
		#pragma unroll
		for (int e = 0; e < PL::EMID; e++) D[(long long)PL::mid(pos, e) * nx + cc] = v[e];
	}
}

template <class K>
cudaError_t smem_attr(K kern, int smem)
{
	if (smem > 48 * 1024) {
		cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
		if (e != cudaSuccess) return e;
	}
	return cudaSuccess;
}

template <class PL>
cudaError_t rows_inv_t(const PgrArgs& p, cudaStream_t s)
{
	constexpr int L = row_lines<PL>();
	constexpr int smem = PL::template smem_elems<RowTileOf<PL>>() * (int)sizeof(float2);
	const dim3 grid((p.ny + L - 1) / L, p.ngr);
	cudaError_t e = smem_attr(k_pgr_rows_inv<PL>, smem);
	if (e != cudaSuccess) return e;
	k_pgr_rows_inv<PL><<<grid, L * PL::TMAX, smem, s>>>(p.out, p.gstride, p.ny, p.twx);
	return cudaGetLastError();
}

template <class PL, int MODE>
cudaError_t cols_mode_t(const PgrArgs& p, const float2* src, float2* dst, cudaStream_t s)
{
	constexpr int C = PL::CC;
	constexpr int smem = PL::template smem_elems<ColTile<C>>() * (int)sizeof(float2);
	const dim3 grid((p.nx + C - 1) / C, p.ngr);
	cudaError_t e = smem_attr(k_pgr_cols<PL, MODE>, smem);
	if (e != cudaSuccess) return e;
	k_pgr_cols<PL, MODE><<<grid, C * PL::TMAX, smem, s>>>(src, dst, p.gstride, p.nx, p.cphase, p.twy);
	return cudaGetLastError();
}

template <class PL>
cudaError_t cols_t(const PgrArgs& p, const float2* src, float2* dst, int mode, cudaStream_t s)
{
	if (mode == kPgrColExpFt) return cols_mode_t<PL, kPgrColExpFt>(p, src, dst, s);
	if (mode == kPgrColExp) return cols_mode_t<PL, kPgrColExp>(p, src, dst, s);
	return cols_mode_t<PL, kPgrColInv>(p, src, dst, s);
}

struct PgrOps {
	int n;
	cudaError_t (*rows_inv)(const PgrArgs&, cudaStream_t);
	cudaError_t (*cols)(const PgrArgs&, const float2*, float2*, int, cudaStream_t);
};
#define JMS_PGR_OPS(n, alias) {n, rows_inv_t<alias>, cols_t<alias>},

// per length group: the default plans' generator transforms, or nullptr
const PgrOps* pgr_ops_0(int n);
const PgrOps* pgr_ops_1(int n);
const PgrOps* pgr_ops_2(int n);

} // namespace jms
