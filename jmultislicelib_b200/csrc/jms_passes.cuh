// jms_passes.cuh -- fused FP32 multislice pass kernels (templates) for sm_100a.
//
// Included by the jms_inst_*.cu files, which instantiate the launchers for
// their share of the supported line lengths; jms_kernels.cu dispatches on the
// grid size.  See jms_kernels.h for the pass structure and jms_fft.cuh for the
// line FFT.  Reference semantics followed here:
//   slice loop order          src/JMultiSlice.cpp:4590-4651 (GPUMultislice)
//   Fourier-space readout     src/JMultiSlice.cpp:4218-4367 (ReadoutDifDet_d)
//   real-space readout        src/JMultiSlice.cpp:4369-4465 (ReadoutImgDet_d)
//   grating multiply          src/cu/ArrayOps.cu:202-234 (MulKernel / sub-frame)
//   probe offset              src/JMultiSlice.cpp:1961-2084, src/cu/ArrayOps.cu:340-421
#pragma once
#include "jms_fft.cuh"
#include "jms_kernels.h"

namespace jms {

// ---------------------------------------------------------------------------
// line transforms with one shared-memory exchange (see jms_fft.cuh)
// ---------------------------------------------------------------------------
// Row tile: LINES rows, thread t -> (line = t / P, pos = t % P) for a role with
// P threads per line; exchange buffer S(line, k1, j) padded to B+1.
template <int LINES>
struct RowTile {
	template <int P>
	__device__ __forceinline__ static void role(int tid, int& line, int& pos) { line = tid / P; pos = tid % P; }
	template <int A, int B>
	__device__ __forceinline__ static int sidx(int line, int k1, int j) { return (line * A + k1) * (B + 1) + j; }
	template <int A, int B>
	static constexpr int sm_elems() { return LINES * A * (B + 1); }
};

// Column tile: C columns, thread t -> (line = t % C, pos = t / C); exchange
// buffer S(c, k1, j) with the column index fastest (padding keeps the k1
// groups of a half warp on distinct banks when C < 16).
template <int C>
struct ColTile {
	static constexpr int PAD = (C < 16) ? C : 0;
	template <int P>
	__device__ __forceinline__ static void role(int tid, int& line, int& pos) { line = tid % C; pos = tid / C; }
	template <int A, int B>
	__device__ __forceinline__ static int sidx(int line, int k1, int j) { return k1 * (B * C + PAD) + j * C + line; }
	template <int A, int B>
	static constexpr int sm_elems() { return A * (B * C + PAD); }
};

// One N = A*B point transform per line.  Input: role with B threads per
// line, thread j holds v[m] = x[j + B m] (m < A).  Output: role with A threads
// per line, thread k1 holds v[k2] = X[k1 + A k2] (k2 < B).  tw = exp(-2 pi i k/N).
// act_in / act_out: this thread's line exists (all threads reach the barriers).
template <int A, int B, bool INV, class Tile, int RM>
__device__ __forceinline__ void line_fft(float2 (&v)[RM], float2* sm, const float2* __restrict__ tw, int tid,
	int nlines_valid)
{
	{
		int line, j;
		Tile::template role<B>(tid, line, j);
		if (line < nlines_valid && j < B) {
			dft_reg<A, 1, 0, INV>(v);
			#pragma unroll
			for (int k1 = 1; k1 < A; k1++) {
				float2 w = __ldg(tw + j * k1); // j*k1 < N
				v[k1] = INV ? cmulc(v[k1], w) : cmul(v[k1], w);
			}
			#pragma unroll
			for (int k1 = 0; k1 < A; k1++) sm[Tile::template sidx<A, B>(line, k1, j)] = v[k1];
		}
	}
	__syncthreads();
	{
		int line, k1;
		Tile::template role<A>(tid, line, k1);
		if (line < nlines_valid && k1 < A) {
			#pragma unroll
			for (int j = 0; j < B; j++) v[j] = sm[Tile::template sidx<A, B>(line, k1, j)];
			dft_reg<B, 1, 0, INV>(v);
		}
	}
	__syncthreads();
}

// ---------------------------------------------------------------------------
// readouts
// ---------------------------------------------------------------------------
__device__ __forceinline__ float warp_sum(float v)
{
	#pragma unroll
	for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
	return v;
}

// Sums acc[d] over the CTA and stores one partial per detector.
template <int NT>
__device__ __forceinline__ void block_store_partials(const float (&acc)[kMaxDet], const PassArgs& p, int b)
{
	__shared__ float red[NT / 32][kMaxDet];
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	#pragma unroll
	for (int d = 0; d < kMaxDet; d++) {
		float s = warp_sum(acc[d]);
		if (lane == 0) red[warp][d] = s;
	}
	__syncthreads();
	if ((int)threadIdx.x < p.ndet) {
		float s = 0.f;
		#pragma unroll
		for (int w = 0; w < NT / 32; w++) s += red[w][threadIdx.x];
		p.partial[(((long long)b * p.ndetslc + p.plane) * p.ndet + threadIdx.x) * p.nblk + blockIdx.x] = s;
	}
	__syncthreads();
}

// Fourier-space readout of one element psi(ky = y, kx) of wave b
// (ReadoutDifDet_d, src/JMultiSlice.cpp:4277-4359).
__device__ __forceinline__ void readout_fourier(const PassArgs& p, int b, int y, int kx, float2 v,
	float (&acc)[kMaxDet])
{
	const long long N = (long long)p.nx * p.ny;
	if (p.descan_x | p.descan_y) {
		// integer-pixel diffraction descan (DescanDifN, src/JMultiSlice.cpp:2184-2273):
		// psi(kx, ky) is read out at pixel (kx - dnx, ky - dny), periodic
		kx -= p.descan_x; kx %= p.nx; if (kx < 0) kx += p.nx;
		y -= p.descan_y; y %= p.ny; if (y < 0) y += p.ny;
	}
	const long long idx = (long long)y * p.nx + kx;
	const float pw = cnorm(v);
	#pragma unroll
	for (int d = 0; d < kMaxDet; d++)
		if (d < p.ndet) acc[d] = fmaf(pw, __ldg(p.det + d * N + idx), acc[d]);
	const long long c = (long long)b * p.chan_wstride + (long long)p.plane * N + idx;
	if (p.dif) p.dif[c] += p.weight * pw;
	if (p.dif_avg) p.dif_avg[c] += p.weight * pw;
	if (p.wff) p.wff[c] = cadd(p.wff[c], cscale(v, p.weight));
	if (p.wff_avg) p.wff_avg[c] = cadd(p.wff_avg[c], cscale(v, p.weight));
	if (p.bin_out && p.plane == p.bin_plane) {
		// unscrambled position (zero beam at nx/2, ny/2 as GetUnscrambleHash,
		// src/JMultiSlice.cpp:1932-1958), then bin x bin pixel blocks
		int ux = kx + (p.nx >> 1); if (ux >= p.nx) ux -= p.nx;
		int uy = y + (p.ny >> 1); if (uy >= p.ny) uy -= p.ny;
		int bx = ux / p.bin, by = uy / p.bin;
		if (bx < p.nbx && by < p.nby)
			atomicAdd(p.bin_out + ((long long)b * p.nby + by) * p.nbx + bx, p.weight * pw);
	}
}

// Real-space readout of psi(y, x) of wave b (ReadoutImgDet_d, src/JMultiSlice.cpp:4392-4459).
__device__ __forceinline__ void readout_real(const PassArgs& p, int b, int y, int x, float2 v)
{
	const long long N = (long long)p.nx * p.ny;
	const long long c = (long long)b * p.chan_wstride + (long long)p.plane * N + (long long)y * p.nx + x;
	const float pw = cnorm(v);
	if (p.img) p.img[c] += p.weight * pw;
	if (p.img_avg) p.img_avg[c] += p.weight * pw;
	if (p.wfr) p.wfr[c] = cadd(p.wfr[c], cscale(v, p.weight));
	if (p.wfr_avg) p.wfr_avg[c] = cadd(p.wfr_avg[c], cscale(v, p.weight));
}

// offset phase plate exp(-i (2 pi turns + cppl)) at scrambled pixel (i, j);
// turns = fi dx/a + fj dy/b + fz (fi^2/a^2 + fj^2/b^2) is formed in FP64 and
// reduced mod 1 before the FP32 sincos (large k.dx phases keep full accuracy).
__device__ __forceinline__ float2 offset_factor(const double* sh, int i, int j, int nx, int ny, float cp)
{
	const int fi = (i + (nx >> 1)) % nx - (nx >> 1);
	const int fj = (j + (ny >> 1)) % ny - (ny >> 1);
	const double di = (double)fi, dj = (double)fj;
	double t = di * sh[0] + dj * sh[1] + di * di * sh[2] + dj * dj * sh[3];
	t -= floor(t);
	float s, c;
	if (cp != 0.f) {
		sincosf(6.283185307179586f * (float)t + cp, &s, &c);
	}
	else {
		sincospif(2.f * (float)t, &s, &c);
	}
	return make_float2(c, -s);
}

// ---------------------------------------------------------------------------
// pass kernels
// ---------------------------------------------------------------------------
template <int R1, int R2>
struct Geo {
	static constexpr int N = R1 * R2;
	static constexpr int RM = R1 > R2 ? R1 : R2;
};

__host__ __device__ constexpr int gcd_ct(int a, int b) { return b == 0 ? a : gcd_ct(b, a % b); }
// rows per row-pass CTA: about 256 threads, thread count a multiple of 32
template <int R1, int R2>
__host__ __device__ constexpr int row_lines()
{
	constexpr int RM = Geo<R1, R2>::RM;
	constexpr int m = 32 / gcd_ct(RM, 32);
	constexpr int l = (256 / RM) / m * m;
	return l < m ? m : l;
}
constexpr int kColC = 16;

// Entry row pass: [offset] -> Fourier readout (plane) -> IFT_x.
template <int R1, int R2>
__global__ void __launch_bounds__(row_lines<R1, R2>() * Geo<R1, R2>::RM)
k_entry_rows(const PassArgs p)
{
	constexpr int N = R1 * R2, RM = Geo<R1, R2>::RM, L = row_lines<R1, R2>(), NT = L * RM;
	using T = RowTile<L>;
	extern __shared__ float2 sm[];
	const int tid = threadIdx.x, b = blockIdx.y, row0 = blockIdx.x * L;
	const int nval = min(L, p.ny - row0);
	float2* W = p.work + (long long)b * p.wstride;
	float2 v[RM];
	float acc[kMaxDet];
	#pragma unroll
	for (int d = 0; d < kMaxDet; d++) acc[d] = 0.f;
	{
		int line, j;
		T::template role<R2>(tid, line, j);
		if (line < nval) {
			const int y = row0 + line;
			#pragma unroll
			for (int m = 0; m < R1; m++) {
				const int kx = j + R2 * m;
				float2 a;
				if (p.shift) {
					int sx = kx - p.ibtx, sy = y - p.ibty;
					sx %= N; if (sx < 0) sx += N;
					sy %= p.ny; if (sy < 0) sy += p.ny;
					a = __ldg(p.wav0 + (long long)sy * N + sx);
					const float cp = p.cppl ? __ldg(p.cppl + (long long)y * N + kx) : 0.f;
					a = cmul(a, offset_factor(p.shift + 4 * b, kx, y, N, p.ny, cp));
				}
				else {
					a = p.wav0 ? __ldg(p.wav0 + (long long)y * N + kx) : W[(long long)y * N + kx];
				}
				if (p.plane >= 0) readout_fourier(p, b, y, kx, a, acc);
				v[m] = a;
			}
		}
	}
	if (p.plane >= 0 && p.ndet > 0) block_store_partials<NT>(acc, p, b);
	line_fft<R1, R2, true, T>(v, sm, p.twx, tid, nval);
	{
		int line, k1;
		T::template role<R1>(tid, line, k1);
		if (line < nval) {
			float2* dst = W + (long long)(row0 + line) * N;
			#pragma unroll
			for (int k2 = 0; k2 < R2; k2++) dst[k1 + R1 * k2] = v[k2];
		}
	}
}

// Row pass: FT_x -> x P -> Fourier readout (plane) -> IFT_x.
template <int R1, int R2>
__global__ void __launch_bounds__(row_lines<R1, R2>() * Geo<R1, R2>::RM)
k_row_pass(const PassArgs p)
{
	constexpr int N = R1 * R2, RM = Geo<R1, R2>::RM, L = row_lines<R1, R2>(), NT = L * RM;
	using T = RowTile<L>;
	extern __shared__ float2 sm[];
	const int tid = threadIdx.x, b = blockIdx.y, row0 = blockIdx.x * L;
	const int nval = min(L, p.ny - row0);
	float2* W = p.work + (long long)b * p.wstride;
	float2 v[RM];
	{
		int line, j;
		T::template role<R2>(tid, line, j);
		if (line < nval) {
			const float2* src = W + (long long)(row0 + line) * N;
			#pragma unroll
			for (int m = 0; m < R1; m++) v[m] = src[j + R2 * m];
		}
	}
	line_fft<R1, R2, false, T>(v, sm, p.twx, tid, nval);
	float acc[kMaxDet];
	#pragma unroll
	for (int d = 0; d < kMaxDet; d++) acc[d] = 0.f;
	{
		int line, k1;
		T::template role<R1>(tid, line, k1);
		if (line < nval) {
			const int y = row0 + line;
			const float2* P = p.mul + (long long)y * N;
			#pragma unroll
			for (int k2 = 0; k2 < R2; k2++) {
				const int kx = k1 + R1 * k2;
				v[k2] = cmul(v[k2], __ldg(P + kx));
				if (p.plane >= 0) readout_fourier(p, b, y, kx, v[k2], acc);
			}
		}
	}
	if (p.plane >= 0 && p.ndet > 0) block_store_partials<NT>(acc, p, b);
	if (!p.store) return;
	line_fft<R2, R1, true, T>(v, sm, p.twx, tid, nval);
	{
		int line, k;
		T::template role<R2>(tid, line, k);
		if (line < nval) {
			float2* dst = W + (long long)(row0 + line) * N;
			#pragma unroll
			for (int k2 = 0; k2 < R1; k2++) dst[k + R2 * k2] = v[k2];
		}
	}
}

// Column pass: IFT_y -> real-space readout (plane) -> x t -> FT_y.
template <int R1, int R2>
__global__ void __launch_bounds__(kColC * Geo<R1, R2>::RM)
k_col_pass(const PassArgs p)
{
	constexpr int N = R1 * R2, RM = Geo<R1, R2>::RM, C = kColC;
	using T = ColTile<C>;
	extern __shared__ float2 sm[];
	const int tid = threadIdx.x, b = blockIdx.y, col0 = blockIdx.x * C;
	const int nval = min(C, p.nx - col0);
	const int nx = p.nx;
	float2* W = p.work + (long long)b * p.wstride + col0;
	float2 v[RM];
	{
		int c, j;
		T::template role<R2>(tid, c, j);
		if (c < nval && j < R2) {
			#pragma unroll
			for (int m = 0; m < R1; m++) v[m] = W[(long long)(j + R2 * m) * nx + c];
		}
	}
	line_fft<R1, R2, true, T>(v, sm, p.twy, tid, nval);
	{
		int c, k1;
		T::template role<R1>(tid, c, k1);
		if (c < nval && k1 < R1) {
			const int x = col0 + c;
			const int xs = x % p.npgx;
			#pragma unroll
			for (int k2 = 0; k2 < R2; k2++) {
				const int y = k1 + R1 * k2;
				if (p.plane >= 0) readout_real(p, b, y, x, v[k2]);
				v[k2] = cmul(v[k2], __ldg(p.mul + (long long)(y % p.npgy) * p.npgx + xs));
			}
		}
	}
	line_fft<R2, R1, false, T>(v, sm, p.twy, tid, nval);
	{
		int c, k;
		T::template role<R2>(tid, c, k);
		if (c < nval && k < R2) {
			#pragma unroll
			for (int k2 = 0; k2 < R1; k2++) W[(long long)(k + R2 * k2) * nx + c] = v[k2];
		}
	}
}

// Exit column pass: IFT_y -> real-space readout (plane), no store.
template <int R1, int R2>
__global__ void __launch_bounds__(kColC * Geo<R1, R2>::RM)
k_exit_cols(const PassArgs p)
{
	constexpr int RM = Geo<R1, R2>::RM, C = kColC;
	using T = ColTile<C>;
	extern __shared__ float2 sm[];
	const int tid = threadIdx.x, b = blockIdx.y, col0 = blockIdx.x * C;
	const int nval = min(C, p.nx - col0);
	const int nx = p.nx;
	const float2* W = p.work + (long long)b * p.wstride + col0;
	float2 v[RM];
	{
		int c, j;
		T::template role<R2>(tid, c, j);
		if (c < nval && j < R2) {
			#pragma unroll
			for (int m = 0; m < R1; m++) v[m] = W[(long long)(j + R2 * m) * nx + c];
		}
	}
	line_fft<R1, R2, true, T>(v, sm, p.twy, tid, nval);
	{
		int c, k1;
		T::template role<R1>(tid, c, k1);
		if (c < nval && k1 < R1) {
			#pragma unroll
			for (int k2 = 0; k2 < R2; k2++) readout_real(p, b, k1 + R1 * k2, col0 + c, v[k2]);
		}
	}
}


// ---------------------------------------------------------------------------
// launchers (explicitly instantiated per size in jms_inst_*.cu)
// ---------------------------------------------------------------------------
template <int R1, int R2>
int row_smem_bytes()
{
	using T = RowTile<row_lines<R1, R2>()>;
	int a = T::template sm_elems<R1, R2>(), b = T::template sm_elems<R2, R1>();
	return (a > b ? a : b) * (int)sizeof(float2);
}
template <int R1, int R2>
int col_smem_bytes()
{
	using T = ColTile<kColC>;
	int a = T::template sm_elems<R1, R2>(), b = T::template sm_elems<R2, R1>();
	return (a > b ? a : b) * (int)sizeof(float2);
}

template <class K>
cudaError_t launch_k(K kern, dim3 grid, int threads, int smem, const PassArgs& p, cudaStream_t s)
{
	static_assert(sizeof(PassArgs) < 4000, "kernel parameter block too large");
	if (smem > 48 * 1024) {
		cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
		if (e != cudaSuccess) return e;
	}
	kern<<<grid, threads, smem, s>>>(p);
	return cudaGetLastError();
}

template <int A, int B>
int row_blocks_t(int ny) { return (ny + row_lines<A, B>() - 1) / row_lines<A, B>(); }

template <int A, int B>
cudaError_t launch_entry_t(const PassArgs& p, cudaStream_t s)
{
	constexpr int L = row_lines<A, B>();
	return launch_k(k_entry_rows<A, B>, dim3((p.ny + L - 1) / L, p.nwave), L * Geo<A, B>::RM, row_smem_bytes<A, B>(), p, s);
}
template <int A, int B>
cudaError_t launch_row_t(const PassArgs& p, cudaStream_t s)
{
	constexpr int L = row_lines<A, B>();
	return launch_k(k_row_pass<A, B>, dim3((p.ny + L - 1) / L, p.nwave), L * Geo<A, B>::RM, row_smem_bytes<A, B>(), p, s);
}
template <int A, int B>
cudaError_t launch_col_t(const PassArgs& p, cudaStream_t s)
{
	return launch_k(k_col_pass<A, B>, dim3((p.nx + kColC - 1) / kColC, p.nwave), kColC * Geo<A, B>::RM,
		col_smem_bytes<A, B>(), p, s);
}
template <int A, int B>
cudaError_t launch_exit_t(const PassArgs& p, cudaStream_t s)
{
	return launch_k(k_exit_cols<A, B>, dim3((p.nx + kColC - 1) / kColC, p.nwave), kColC * Geo<A, B>::RM,
		col_smem_bytes<A, B>(), p, s);
}

#define JMS_INSTANTIATE(A, B) \
	template int row_blocks_t<A, B>(int); \
	template cudaError_t launch_entry_t<A, B>(const PassArgs&, cudaStream_t); \
	template cudaError_t launch_row_t<A, B>(const PassArgs&, cudaStream_t); \
	template cudaError_t launch_col_t<A, B>(const PassArgs&, cudaStream_t); \
	template cudaError_t launch_exit_t<A, B>(const PassArgs&, cudaStream_t);

} // namespace jms
