// jms_nn.cu -- kernels of the control-variate surrogate network (BF16
// storage, FP32 accumulation), training and inference.
//
// The surrogate maps a local projected-potential patch around the probe
// (one channel per depth bin) to the integrated detector signals at the
// readout thicknesses.  Layers: 3x3 convolutions of stride 2 and padding 1,
// with or without ReLU (BF16 activations and weights), a global average pool,
// and a linear layer (FP32).  The host side (jmultislicelib_b200/surrogate.py)
// owns the buffers and the training loop; these kernels are the building
// blocks: forward, both backward products, loss, Adam.
//
// Layouts: activations [B][C][H][W]; conv weights [Co][Ci][3][3]; linear
// weights [O][C].  The ReLU mask of a layer is its stored output (y > 0).
#include "../../include/jms_b200.h"

#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace {

__device__ __forceinline__ float bf(const __nv_bfloat16 v) { return __bfloat162float(v); }

// y[b][co][oy][ox] = relu(bias[co] + sum_ci,ky,kx w[co][ci][ky][kx] x[b][ci][2oy-1+ky][2ox-1+kx])
__global__ void k_conv_fwd(const __nv_bfloat16* __restrict__ x, const __nv_bfloat16* __restrict__ w,
	const float* __restrict__ bias, __nv_bfloat16* __restrict__ y, int B, int Ci, int H, int W, int Co, int relu)
{
	const int Ho = H / 2, Wo = W / 2;
	const long long n = (long long)B * Co * Ho * Wo;
	const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	const int ox = (int)(i % Wo), oy = (int)((i / Wo) % Ho), co = (int)((i / ((long long)Wo * Ho)) % Co);
	const int b = (int)(i / ((long long)Wo * Ho * Co));
	float acc = bias[co];
	for (int ci = 0; ci < Ci; ci++) {
		const __nv_bfloat16* xp = x + ((long long)b * Ci + ci) * H * W;
		const __nv_bfloat16* wp = w + ((long long)co * Ci + ci) * 9;
		#pragma unroll
		for (int ky = 0; ky < 3; ky++) {
			const int iy = 2 * oy - 1 + ky;
			if (iy < 0 || iy >= H) continue;
			#pragma unroll
			for (int kx = 0; kx < 3; kx++) {
				const int ix = 2 * ox - 1 + kx;
				if (ix < 0 || ix >= W) continue;
				acc = fmaf(bf(wp[ky * 3 + kx]), bf(xp[iy * W + ix]), acc);
			}
		}
	}
	if (relu && acc < 0.f) acc = 0.f;
	y[i] = __float2bfloat16(acc);
}

// dx[b][ci][iy][ix] = sum_co,ky,kx g[b][co][oy][ox] w[co][ci][ky][kx], iy = 2oy-1+ky,
// with g = dy * (y > 0) when relu
__global__ void k_conv_bwd_data(const float* __restrict__ dy, const __nv_bfloat16* __restrict__ y,
	const __nv_bfloat16* __restrict__ w, float* __restrict__ dx, int B, int Ci, int H, int W, int Co, int relu)
{
	const int Ho = H / 2, Wo = W / 2;
	const long long n = (long long)B * Ci * H * W;
	const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	const int ix = (int)(i % W), iy = (int)((i / W) % H), ci = (int)((i / ((long long)W * H)) % Ci);
	const int b = (int)(i / ((long long)W * H * Ci));
	float acc = 0.f;
	#pragma unroll
	for (int ky = 0; ky < 3; ky++) {
		const int t = iy + 1 - ky;                   // = 2 oy
		if (t < 0 || (t & 1)) continue;
		const int oy = t >> 1;
		if (oy >= Ho) continue;
		#pragma unroll
		for (int kx = 0; kx < 3; kx++) {
			const int u = ix + 1 - kx;
			if (u < 0 || (u & 1)) continue;
			const int ox = u >> 1;
			if (ox >= Wo) continue;
			for (int co = 0; co < Co; co++) {
				const long long o = (((long long)b * Co + co) * Ho + oy) * Wo + ox;
				float g = dy[o];
				if (relu && !(bf(y[o]) > 0.f)) g = 0.f;
				acc = fmaf(g, bf(w[((long long)co * Ci + ci) * 9 + ky * 3 + kx]), acc);
			}
		}
	}
	dx[i] = acc;
}

// dw[co][ci][ky][kx] = sum_b,oy,ox g[b][co][oy][ox] x[b][ci][iy][ix]; db[co] = sum g.
// One CTA per (co, ci) with a block reduction; ci = Ci is the bias slot.
__global__ void __launch_bounds__(256) k_conv_bwd_weight(const __nv_bfloat16* __restrict__ x,
	const float* __restrict__ dy, const __nv_bfloat16* __restrict__ y, float* __restrict__ dw, float* __restrict__ db,
	int B, int Ci, int H, int W, int Co, int relu)
{
	const int co = blockIdx.x / (Ci + 1), ci = blockIdx.x % (Ci + 1);
	const int Ho = H / 2, Wo = W / 2;
	const long long n = (long long)B * Ho * Wo;
	float acc[9];
	#pragma unroll
	for (int k = 0; k < 9; k++) acc[k] = 0.f;
	for (long long i = threadIdx.x; i < n; i += blockDim.x) {
		const int ox = (int)(i % Wo), oy = (int)((i / Wo) % Ho), b = (int)(i / ((long long)Wo * Ho));
		const long long o = (((long long)b * Co + co) * Ho + oy) * Wo + ox;
		float g = dy[o];
		if (relu && !(bf(y[o]) > 0.f)) g = 0.f;
		if (ci == Ci) { acc[0] += g; continue; }
		const __nv_bfloat16* xp = x + ((long long)b * Ci + ci) * H * W;
		#pragma unroll
		for (int ky = 0; ky < 3; ky++) {
			const int iy = 2 * oy - 1 + ky;
			if (iy < 0 || iy >= H) continue;
			#pragma unroll
			for (int kx = 0; kx < 3; kx++) {
				const int ix = 2 * ox - 1 + kx;
				if (ix < 0 || ix >= W) continue;
				acc[ky * 3 + kx] = fmaf(g, bf(xp[iy * W + ix]), acc[ky * 3 + kx]);
			}
		}
	}
	__shared__ float red[9][8];
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	#pragma unroll
	for (int k = 0; k < 9; k++) {
		float v = acc[k];
		#pragma unroll
		for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
		if (lane == 0) red[k][warp] = v;
	}
	__syncthreads();
	if (threadIdx.x < 9) {
		float v = 0.f;
		for (int k = 0; k < (int)(blockDim.x >> 5); k++) v += red[threadIdx.x][k];
		if (ci == Ci) { if (threadIdx.x == 0) db[co] = v; }
		else dw[((long long)co * Ci + ci) * 9 + threadIdx.x] = v;
	}
}

// out[b][o] = bl[o] + sum_c wl[o][c] mean_hw h[b][c][hw]
__global__ void k_pool_linear_fwd(const __nv_bfloat16* __restrict__ h, const float* __restrict__ wl,
	const float* __restrict__ bl, float* __restrict__ out, int B, int C, int HW, int O)
{
	extern __shared__ float pooled[];   // [C]
	const int b = blockIdx.x;
	for (int c = threadIdx.x; c < C; c += blockDim.x) {
		const __nv_bfloat16* hp = h + ((long long)b * C + c) * HW;
		float s = 0.f;
		for (int k = 0; k < HW; k++) s += bf(hp[k]);
		pooled[c] = s / (float)HW;
	}
	__syncthreads();
	for (int o = threadIdx.x; o < O; o += blockDim.x) {
		float s = bl[o];
		for (int c = 0; c < C; c++) s = fmaf(wl[(long long)o * C + c], pooled[c], s);
		out[(long long)b * O + o] = s;
	}
}

// dh[b][c][hw] = sum_o dout[b][o] wl[o][c] / HW; dwl, dbl by a second kernel
__global__ void k_pool_linear_bwd_data(const float* __restrict__ wl, const float* __restrict__ dout,
	float* __restrict__ dh, int B, int C, int HW, int O)
{
	const long long n = (long long)B * C * HW;
	const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	const int c = (int)((i / HW) % C), b = (int)(i / ((long long)HW * C));
	float s = 0.f;
	for (int o = 0; o < O; o++) s = fmaf(dout[(long long)b * O + o], wl[(long long)o * C + c], s);
	dh[i] = s / (float)HW;
}

// dwl[o][c] = sum_b dout[b][o] pooled[b][c]; dbl[o] = sum_b dout[b][o]; thread per (o, c | bias)
__global__ void k_pool_linear_bwd_weight(const __nv_bfloat16* __restrict__ h, const float* __restrict__ dout,
	float* __restrict__ dwl, float* __restrict__ dbl, int B, int C, int HW, int O)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= O * (C + 1)) return;
	const int o = i / (C + 1), c = i % (C + 1);
	float s = 0.f;
	for (int b = 0; b < B; b++) {
		const float g = dout[(long long)b * O + o];
		if (c == C) { s += g; continue; }
		const __nv_bfloat16* hp = h + ((long long)b * C + c) * HW;
		float p = 0.f;
		for (int k = 0; k < HW; k++) p += bf(hp[k]);
		s = fmaf(g, p / (float)HW, s);
	}
	if (c == C) dbl[o] = s;
	else dwl[(long long)o * C + c] = s;
}

// dout = 2 (out - t) / n; loss partial sums of (out - t)^2 / n (atomic into *loss)
__global__ void k_mse(const float* __restrict__ out, const float* __restrict__ t, float* __restrict__ dout,
	float* __restrict__ loss, int n)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	float e = 0.f;
	if (i < n) {
		const float d = out[i] - t[i];
		dout[i] = 2.f * d / (float)n;
		e = d * d / (float)n;
	}
	#pragma unroll
	for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(0xffffffffu, e, o);
	if ((threadIdx.x & 31) == 0 && loss) atomicAdd(loss, e);
}

// Adam (Kingma & Ba 2015) on FP32 master weights, optional BF16 copy.
__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
	float* __restrict__ v, __nv_bfloat16* __restrict__ pb, int n, float lr, float b1, float b2, float eps,
	float c1, float c2)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	const float gi = g[i];
	const float mi = b1 * m[i] + (1.f - b1) * gi;
	const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
	m[i] = mi;
	v[i] = vi;
	const float pi = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
	p[i] = pi;
	if (pb) pb[i] = __float2bfloat16(pi);
}

__global__ void k_cast_bf16(const float* __restrict__ s, __nv_bfloat16* __restrict__ d, long long n)
{
	const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) d[i] = __float2bfloat16(s[i]);
}

inline unsigned nblk(long long n, int t) { return (unsigned)((n + t - 1) / t); }

// Surrogate inputs: thread per output value out[c][p][b][u][v], the mean over
// the object slices of depth bin b (bins of nobj / nbins slices, the first
// nobj % nbins one slice longer) and over a pool x pool pixel block of the
// projected potential of configuration c, in the win x win window centred on
// pixel (px, py) of position p (periodic).
__global__ void k_patches(const float* __restrict__ pot, int nvar, int nx, int ny, const int* __restrict__ objslc,
	int nobj, const int* __restrict__ var, int nconf, const int* __restrict__ pix, int npos, int nbins, int win,
	int pool, float* __restrict__ out)
{
	const int m = win / pool;
	const long long n = (long long)nconf * npos * nbins * m * m;
	const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	const int v = (int)(i % m), u = (int)((i / m) % m);
	const int b = (int)((i / ((long long)m * m)) % nbins);
	const int p = (int)((i / ((long long)m * m * nbins)) % npos);
	const int c = (int)(i / ((long long)m * m * nbins * npos));
	const int q = nobj / nbins, r = nobj % nbins;
	const int s0 = b * q + min(b, r), s1 = s0 + q + (b < r ? 1 : 0);
	const int x0 = pix[2 * p] - win / 2 + v * pool, y0 = pix[2 * p + 1] - win / 2 + u * pool;
	const long long N = (long long)nx * ny;
	float acc = 0.f;
	for (int s = s0; s < s1; s++) {
		const float* map = pot + ((long long)objslc[s] * nvar + var[(long long)c * nobj + s]) * N;
		for (int dy = 0; dy < pool; dy++) {
			int y = (y0 + dy) % ny;
			if (y < 0) y += ny;
			for (int dx = 0; dx < pool; dx++) {
				int x = (x0 + dx) % nx;
				if (x < 0) x += nx;
				acc += __ldg(map + (long long)y * nx + x);
			}
		}
	}
	out[i] = acc / (float)((s1 - s0) * pool * pool);
}
inline int ok(cudaStream_t) { return cudaGetLastError() == cudaSuccess ? 0 : 1; }

} // namespace

extern "C" {

int JMS_NnConvForward(const void* x, const void* w, const float* bias, void* y, int B, int Ci, int H, int W, int Co,
	int relu, void* stream)
{
	if (!x || !w || !bias || !y || B < 1 || Ci < 1 || Co < 1 || H < 2 || W < 2 || (H & 1) || (W & 1)) return 2;
	cudaStream_t s = (cudaStream_t)stream;
	const long long n = (long long)B * Co * (H / 2) * (W / 2);
	k_conv_fwd<<<nblk(n, 256), 256, 0, s>>>((const __nv_bfloat16*)x, (const __nv_bfloat16*)w, bias,
		(__nv_bfloat16*)y, B, Ci, H, W, Co, relu);
	return ok(s);
}

int JMS_NnConvBackward(const void* x, const void* w, const void* y, const float* dy, float* dx, float* dw, float* db,
	int B, int Ci, int H, int W, int Co, int relu, void* stream)
{
	if (!x || !w || !y || !dy || !dw || !db || B < 1 || Ci < 1 || Co < 1 || (H & 1) || (W & 1)) return 2;
	cudaStream_t s = (cudaStream_t)stream;
	if (dx) {
		const long long n = (long long)B * Ci * H * W;
		k_conv_bwd_data<<<nblk(n, 256), 256, 0, s>>>(dy, (const __nv_bfloat16*)y, (const __nv_bfloat16*)w, dx, B, Ci,
			H, W, Co, relu);
	}
	k_conv_bwd_weight<<<(unsigned)(Co * (Ci + 1)), 256, 0, s>>>((const __nv_bfloat16*)x, dy, (const __nv_bfloat16*)y,
		dw, db, B, Ci, H, W, Co, relu);
	return ok(s);
}

int JMS_NnPoolLinearForward(const void* h, const float* wl, const float* bl, float* out, int B, int C, int HW, int O,
	void* stream)
{
	if (!h || !wl || !bl || !out || B < 1 || C < 1 || HW < 1 || O < 1 || C > 8192) return 2;
	cudaStream_t s = (cudaStream_t)stream;
	k_pool_linear_fwd<<<(unsigned)B, 128, sizeof(float) * C, s>>>((const __nv_bfloat16*)h, wl, bl, out, B, C, HW, O);
	return ok(s);
}

int JMS_NnPoolLinearBackward(const void* h, const float* wl, const float* dout, float* dh, float* dwl, float* dbl,
	int B, int C, int HW, int O, void* stream)
{
	if (!h || !wl || !dout || !dwl || !dbl || B < 1 || C < 1 || HW < 1 || O < 1) return 2;
	cudaStream_t s = (cudaStream_t)stream;
	if (dh) {
		const long long n = (long long)B * C * HW;
		k_pool_linear_bwd_data<<<nblk(n, 256), 256, 0, s>>>(wl, dout, dh, B, C, HW, O);
	}
	k_pool_linear_bwd_weight<<<nblk((long long)O * (C + 1), 128), 128, 0, s>>>((const __nv_bfloat16*)h, dout, dwl, dbl,
		B, C, HW, O);
	return ok(s);
}

int JMS_NnMseLoss(const float* out, const float* target, float* dout, float* loss, int n, void* stream)
{
	if (!out || !target || !dout || n < 1) return 2;
	cudaStream_t s = (cudaStream_t)stream;
	if (loss) cudaMemsetAsync(loss, 0, sizeof(float), s);
	k_mse<<<nblk(n, 256), 256, 0, s>>>(out, target, dout, loss, n);
	return ok(s);
}

int JMS_NnAdam(float* p, const float* g, float* m, float* v, void* p_bf16, int n, float lr, float b1, float b2,
	float eps, int step, void* stream)
{
	if (!p || !g || !m || !v || n < 1 || step < 1) return 2;
	cudaStream_t s = (cudaStream_t)stream;
	const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
	k_adam<<<nblk(n, 256), 256, 0, s>>>(p, g, m, v, (__nv_bfloat16*)p_bf16, n, lr, b1, b2, eps, c1, c2);
	return ok(s);
}

int JMS_NnPatches(const float* pot, int ntype, int nvar, int nx, int ny, const int* objslc, int nobj, const int* var,
	int nconf, const int* pix, int npos, int nbins, int win, int pool, float* out, void* stream)
{
	if (!pot || !objslc || !var || !pix || !out || ntype < 1 || nvar < 1 || nx < 1 || ny < 1 || nobj < 1 ||
		nconf < 1 || npos < 1 || nbins < 1 || nbins > nobj || win < 1 || pool < 1 || win % pool)
		return 2;
	cudaStream_t s = (cudaStream_t)stream;
	const long long m = win / pool, n = (long long)nconf * npos * nbins * m * m;
	k_patches<<<nblk(n, 256), 256, 0, s>>>(pot, nvar, nx, ny, objslc, nobj, var, nconf, pix, npos, nbins, win, pool,
		out);
	return ok(s);
}

int JMS_NnCastBf16(const float* src, void* dst, long long n, void* stream)
{
	if (!src || !dst || n < 1) return 2;
	cudaStream_t s = (cudaStream_t)stream;
	k_cast_bf16<<<nblk(n, 256), 256, 0, s>>>(src, (__nv_bfloat16*)dst, n);
	return ok(s);
}

} // extern "C"
