// jms_noalloc.cu -- integrated-detector readout that allocates no memory.
//
// Some callers cannot let a library allocate device memory while they run:
// a program that has already handed the whole GPU to a fixed memory pool, a
// real-time loop that must not stall (cudaMalloc and cudaFree synchronise the
// device), or a host application that has to keep its memory footprint
// fixed after start-up.  For them this file provides a variant of the
// Fourier-space detector readout of the row pass: the per-CTA partial sums,
// which the regular path keeps in a buffer the library allocates, live here
// in one file-scope device array of fixed size, and the caller supplies the
// wave and the output.
//
// Limits and rules (also stated at the declaration in include/jms_b200.h):
//   - the scratch array holds kNoAllocPartials floats (256 KiB); a call needs
//     nwave * ndet * ceil(ny / 8) of them and is refused beyond that;
//   - every GPU that loads the library holds the array until the process ends;
//   - all calls share the array: calls whose work overlaps on the GPU (for
//     example from two streams) race on it;
//   - the first call on a device looks up the array's device address with
//     cudaGetSymbolAddress while that device is current; make that first call
//     before any stream capture.  Later calls on the device reuse the address
//     as long as the same CUDA context is current there; a call under another
//     context of that device (after cudaDeviceReset, or a caller-made
//     context) looks the address up again;
//   - JMS_ReadoutDetAvg with JMS_DETECT_INTEGRATED uses the same array on the
//     library's stream, so callers serialise it with calls of this entry point
//     on other streams.
// Every partial sum the reduction reads is written earlier in the same call,
// so nothing has to be cleared between calls.
#include "jms_kernels.h"

#include <cuda.h>
#include <cstdio>
#include <mutex>

namespace jms {

constexpr int kNoAllocPartials = 65536;
constexpr int kNoAllocRows = 8;        // rows per CTA of the readout kernel
constexpr int kNoAllocThreads = 256;
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) float g_noalloc_partial[kNoAllocPartials];

// One CTA reads kNoAllocRows rows of one wave, accumulates |psi(k)|^2 D_d(k)
// for every detector, and stores one partial sum per detector.
__global__ void __launch_bounds__(kNoAllocThreads)
k_readout_noalloc(const float2* __restrict__ wav, int nx, int ny, const float* __restrict__ det, int ndet,
	float* __restrict__ partial, int nblk)
{
	const int b = blockIdx.y;
	const long long N = (long long)nx * ny;
	const int row0 = blockIdx.x * kNoAllocRows;
	const int nrow = min(kNoAllocRows, ny - row0);
	const float2* w = wav + (long long)b * N + (long long)row0 * nx;
	const float* dd = det + (long long)row0 * nx;
	float acc[kMaxDet];
	#pragma unroll
	for (int d = 0; d < kMaxDet; d++) acc[d] = 0.f;
	const int n = nrow * nx;
	for (int i = threadIdx.x; i < n; i += kNoAllocThreads) {
		const float2 v = w[i];
		const float pw = fmaf(v.x, v.x, v.y * v.y);
		#pragma unroll
		for (int d = 0; d < kMaxDet; d++)
			if (d < ndet) acc[d] = fmaf(pw, __ldg(dd + d * N + i), acc[d]);
	}
	__shared__ float red[kNoAllocThreads / 32][kMaxDet];
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	#pragma unroll
	for (int d = 0; d < kMaxDet; d++) {
		float s = acc[d];
		#pragma unroll
		for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
		if (lane == 0) red[warp][d] = s;
	}
	__syncthreads();
	if ((int)threadIdx.x < ndet) {
		float s = 0.f;
		#pragma unroll
		for (int k = 0; k < kNoAllocThreads / 32; k++) s += red[k][threadIdx.x];
		partial[((long long)b * ndet + threadIdx.x) * nblk + blockIdx.x] = s;
	}
}

// out[w][d] = sum over the CTAs of the partial sums (FP64); overwrites out.
__global__ void k_reduce_noalloc(const float* __restrict__ partial, int n, int nblk, double* out)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	double s = 0.0;
	for (int k = 0; k < nblk; k++) s += (double)partial[(long long)i * nblk + k];
	out[i] = s;
}

// The driver context current on the calling thread (nullptr if none or if the
// driver entry point is unavailable), through the runtime's driver entry-point
// query, so the library needs no link to the driver library.
static CUcontext current_context()
{
	typedef CUresult (*GetCurrent)(CUcontext*);
	static GetCurrent fn = nullptr;
	static std::once_flag once;
	std::call_once(once, []() {
		void* f = nullptr;
		cudaDriverEntryPointQueryResult q;
		if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
			q == cudaDriverEntryPointSuccess)
			fn = (GetCurrent)f;
	});
	CUcontext c = nullptr;
	if (fn == nullptr || fn(&c) != CUDA_SUCCESS) return nullptr;
	return c;
}

// Device address of the scratch array on the current device, looked up once
// per device and context (cudaGetSymbolAddress; host code cannot use the
// symbol itself, and the address belongs to the context it was made in).
static int noalloc_scratch(float** ptr)
{
	static std::mutex mu;
	static float* addr[kNoAllocMaxDevices] = {nullptr};
	static CUcontext owner[kNoAllocMaxDevices] = {nullptr};
	int dev = -1;
	if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNoAllocMaxDevices) return 1;
	const CUcontext ctx = current_context();
	std::lock_guard<std::mutex> lock(mu);
	if (addr[dev] == nullptr || owner[dev] != ctx) {
		void* p = nullptr;
		const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_partial);
		if (e != cudaSuccess || p == nullptr) {
			std::fprintf(stderr, "Error: (ReadoutDetectorsNoAlloc): no device address for the scratch array: %s\n",
				cudaGetErrorString(e));
			return 2;
		}
		addr[dev] = (float*)p;
		owner[dev] = current_context();   // the context the lookup ran in (made current by it if none was)
	}
	*ptr = addr[dev];
	return 0;
}

int noalloc_capacity() { return kNoAllocPartials; }

int launch_readout_noalloc(const float2* wav, int nwave, int nx, int ny, const float* det, int ndet, double* out,
	cudaStream_t s)
{
	const int nblk = (ny + kNoAllocRows - 1) / kNoAllocRows;
	if ((long long)nwave * ndet * nblk > kNoAllocPartials) return 131;
	float* scratch = nullptr;
	if (noalloc_scratch(&scratch)) return 132;
	k_readout_noalloc<<<dim3(nblk, nwave), kNoAllocThreads, 0, s>>>(wav, nx, ny, det, ndet, scratch, nblk);
	if (cudaGetLastError() != cudaSuccess) return 133;
	const int n = nwave * ndet;
	k_reduce_noalloc<<<(n + 127) / 128, 128, 0, s>>>(scratch, n, nblk, out);
	if (cudaGetLastError() != cudaSuccess) return 133;
	return 0;
}

} // namespace jms
