// jms_kernels.cu -- size dispatch and the small kernels of the library
// (per-run detector reduction, probe offset, scan offsets).
#include "jms_fft.cuh"
#include "jms_kernels.h"
#include "jms_sizes.h"

namespace jms {

__device__ __forceinline__ float2 offset_factor_k(const double* sh, int i, int j, int nx, int ny, float cp)
{
	const int fi = (i + (nx >> 1)) % nx - (nx >> 1);
	const int fj = (j + (ny >> 1)) % ny - (ny >> 1);
	const double di = (double)fi, dj = (double)fj;
	double t = di * sh[0] + dj * sh[1] + di * di * sh[2] + dj * dj * sh[3];
	t -= floor(t);
	float s, c;
	if (cp != 0.f) sincosf(6.283185307179586f * (float)t + cp, &s, &c);
	else sincospif(2.f * (float)t, &s, &c);
	return make_float2(c, -s);
}

__global__ void k_make_shift(double* sh, const float* __restrict__ pos, int npos, double a, double b, double fz)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= npos) return;
	sh[4 * i + 0] = (double)pos[2 * i] / a;
	sh[4 * i + 1] = (double)pos[2 * i + 1] / b;
	sh[4 * i + 2] = fz / (a * a);
	sh[4 * i + 3] = fz / (b * b);
}

__global__ void k_abs2(float* __restrict__ out, const float2* __restrict__ in, long long n)
{
	const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	const float2 v = in[i];
	out[i] = v.x * v.x + v.y * v.y;
}

__global__ void k_cv_combine(double* __restrict__ out, const double* __restrict__ g1, const double* __restrict__ gm,
	long long n, double c)
{
	const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) out[i] += c * (gm[i] - g1[i]);
}

cudaError_t launch_cv_combine(double* out, const double* g1, const double* gm, long long n, double c, cudaStream_t s)
{
	if (n <= 0) return cudaSuccess;
	k_cv_combine<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(out, g1, gm, n, c);
	return cudaGetLastError();
}

// thread i = (position p, plane, detector) of n outputs; m = ndetslc * ndet
// elements per wave; the waves of position p are p + k * step, k < nk
__global__ void k_finalize(const float* __restrict__ partial, int n, int m, int nblk, int step, int nk, float weight,
	double* det_int)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	const int pos = i / m, e = i - pos * m;
	double s = 0.0;
	for (int k = 0; k < nk; k++) {
		const float* src = partial + ((long long)(pos + k * step) * m + e) * nblk;
		for (int b = 0; b < nblk; b++) s += (double)src[b];
	}
	det_int[i] += (double)weight * s;
}

__global__ void k_gather_shift(double* __restrict__ sh_w, const double* __restrict__ sh, int npos, int nwave)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= 4 * nwave) return;
	const int w = i >> 2, c = i & 3;
	sh_w[i] = sh[4 * (w % npos) + c];
}

cudaError_t launch_gather_shift(double* sh_w, const double* sh, int npos, int nwave, cudaStream_t s)
{
	if (nwave <= 0 || npos <= 0) return cudaSuccess;
	k_gather_shift<<<(4 * nwave + 255) / 256, 256, 0, s>>>(sh_w, sh, npos, nwave);
	return cudaGetLastError();
}

__global__ void k_offset(float2* out, const float2* __restrict__ wav0, int nx, int ny, double s0, double s1,
	double s2, double s3, const float* __restrict__ cppl, int ibtx, int ibty)
{
	const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	if (idx >= (long long)nx * ny) return;
	const int i = (int)(idx % nx), j = (int)(idx / nx);
	const double sh[4] = {s0, s1, s2, s3};
	int sx = (i - ibtx) % nx; if (sx < 0) sx += nx;
	int sy = (j - ibty) % ny; if (sy < 0) sy += ny;
	const float cp = cppl ? cppl[idx] : 0.f;
	out[idx] = cmul(wav0[(long long)sy * nx + sx], offset_factor_k(sh, i, j, nx, ny, cp));
}


// ---------------------------------------------------------------------------
// plan table
// ---------------------------------------------------------------------------
static const PlanOps kPlans[] = {
#define X(n_, pl_, name_) {n_, name_, &row_blocks_t<pl_>, &launch_entry_t<pl_>, &launch_row_t<pl_>, \
	&launch_col_t<pl_>, &launch_exit_t<pl_>},
	JMS_PLANS(X)
#undef X
};
static constexpr int kNumPlans = (int)(sizeof(kPlans) / sizeof(kPlans[0]));

int plan_count(int n)
{
	int c = 0;
	for (int i = 0; i < kNumPlans; i++) c += (kPlans[i].n == n);
	return c;
}

const PlanOps* plan_get(int n, int idx)
{
	for (int i = 0; i < kNumPlans; i++)
		if (kPlans[i].n == n && idx-- == 0) return &kPlans[i];
	return nullptr;
}

cudaError_t launch_finalize(const float* partial, int nwave, int ndetslc, int ndet, int nblk, float weight,
	double* det_int, cudaStream_t s, int wave_pos)
{
	const int m = ndetslc * ndet;
	const int npos = wave_pos > 0 ? wave_pos : nwave;
	const int nk = wave_pos > 0 ? nwave / wave_pos : 1;
	const int n = npos * m;
	if (n <= 0) return cudaSuccess;
	k_finalize<<<(n + 255) / 256, 256, 0, s>>>(partial, n, m, nblk, npos, nk, weight, det_int);
	return cudaGetLastError();
}

cudaError_t launch_make_shift(double* d_shift, const float* d_pos, int npos, double a, double b, double fz,
	cudaStream_t s)
{
	k_make_shift<<<(npos + 127) / 128, 128, 0, s>>>(d_shift, d_pos, npos, a, b, fz);
	return cudaGetLastError();
}

cudaError_t launch_abs2(float* out, const float2* in, long long n, cudaStream_t s)
{
	if (n <= 0) return cudaSuccess;
	k_abs2<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(out, in, n);
	return cudaGetLastError();
}

cudaError_t launch_offset(float2* out, const float2* wav0, int nx, int ny, const double* sh, const float* cppl,
	int ibtx, int ibty, cudaStream_t s)
{
	const long long n = (long long)nx * ny;
	k_offset<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(out, wav0, nx, ny, sh[0], sh[1], sh[2], sh[3], cppl,
		ibtx, ibty);
	return cudaGetLastError();
}

} // namespace jms
