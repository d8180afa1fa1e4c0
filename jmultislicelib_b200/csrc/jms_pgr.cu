// jms_pgr.cu -- kernels of the on-device phase-grating generator (jms_pgr.h).
#include "jms_pgr_t.cuh"

namespace jms {

// ---------------------------------------------------------------------------
// site displacements (quantum excitation of phonons)
// ---------------------------------------------------------------------------
// SplitMix64 (Steele, Lea, Flood, OOPSLA 2014): state_k = seed + k * gamma,
// output = mix(state_k).  Draw pair c of grating g, site s uses k = 2c + 1 and
// 2c + 2 with c = g * nsite + s.
__device__ __forceinline__ unsigned long long sm64(unsigned long long seed, unsigned long long k)
{
	unsigned long long z = seed + k * 0x9E3779B97F4A7C15ull;
	z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
	z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
	return z ^ (z >> 31);
}

__global__ void k_pgr_sites(double2* pos, const double2* base, const double* uxf, const double* uyf, int nsite,
	int ngr, unsigned long long seed)
{
	const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= (long long)nsite * ngr) return;
	const int s = (int)(i % nsite);
	double2 p = base[s];
	if (uxf[s] != 0.0 || uyf[s] != 0.0) {
		const unsigned long long c = (unsigned long long)i;
		const double u1 = (double)((sm64(seed, 2 * c + 1) >> 11) + 1) * 0x1.0p-53;   // (0, 1]
		const double u2 = (double)(sm64(seed, 2 * c + 2) >> 11) * 0x1.0p-53;         // [0, 1)
		const double r = sqrt(-2.0 * log(u1));
		double sn, cs;
		sincospi(2.0 * u2, &sn, &cs);
		p.x += uxf[s] * r * cs;
		p.y += uyf[s] * r * sn;
	}
	pos[i] = p;
}

cudaError_t launch_pgr_sites(double2* pos, const double2* base, const double* ux_frac, const double* uy_frac,
	int nsite, int ngr, unsigned long long seed, cudaStream_t s)
{
	const long long n = (long long)nsite * ngr;
	if (n <= 0) return cudaSuccess;
	k_pgr_sites<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(pos, base, ux_frac, uy_frac, nsite, ngr, seed);
	return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Fourier synthesis of the projected potential
// ---------------------------------------------------------------------------
// The structure factor S_t(q) = sum_a occ_a exp(-2 pi i (x_a qx + y_a qy))
// is separable per atom, exp(-2 pi i (x qx + y qy)) = ex(qx) ey(qy), so the
// synthesis runs on tables made once per call:
//   k_pgr_phase: ex of every atom and column, occ * ey of every atom and row,
//                the phase in turns x/a * fi formed in FP64 and reduced to
//                [-1/2, 1/2) before the FP32 sincospi;
//   k_pgr_fq:    f_t(|q|) (times ap(q)^2 under bwl_pot) of every type and
//                pixel, once per setup;
//   k_pgr_synth: a CTA owns a 64 x 64 pixel tile of one grating; thread
//                (lane, warp) keeps S of columns 2 lane, 2 lane + 1 and rows
//                8 warp ... +7 in registers (64 FMAs per atom against 5
//                shared loads).  Real occupancies make S Hermitian,
//                S(-q) = conj(S(q)): tiles cover rows iy < ceil(ny / 2) and
//                also write f_t conj(S_t) at the mirrored pixel
//                (ny - iy, (nx - ix) mod nx);
//   k_pgr_lines: the pixels without a sampled mirror, summed directly from
//                the same tables: the Nyquist row ny / 2 (even ny) and the
//                Nyquist column nx / 2 of the mirrored rows (even nx), where
//                the grid samples -n/2 and not its partner +n/2.
// Every output sums its atoms in type order, then atom order, with two FMAs
// per component and atom, and adds f_t S_t over the types in order.
namespace {
constexpr int kSX = 64, kSY = 64, kRW = 8, kCH = 16, kSThr = 256;
constexpr int kChunkF2 = kCH * (kSX + kSY);     // float2 per staged chunk: ex [kCH][kSX], then ey [kCH][kSY]

// signed frequency index of bin i < n: 0, 1, ..., then -floor(n/2), ..., -1
__device__ __forceinline__ int freq(int i, int n)
{
	return i < n - (n >> 1) ? i : i - n;
}

__device__ __forceinline__ float2 cis_turns_neg(double t)
{
	t -= rint(t);
	float s, c;
	sincospif(2.f * (float)t, &s, &c);
	return make_float2(c, -s);
}

// S += e * w (complex)
__device__ __forceinline__ void cmac(float2& S, float ex, float ey, float wx, float wy)
{
	S.x = fmaf(ex, wx, fmaf(-ey, wy, S.x));
	S.y = fmaf(ex, wy, fmaf(ey, wx, S.y));
}

// 8-byte asynchronous copy global -> shared; valid = false writes zeros
// (cp_async_commit: jms_passes.cuh)
__device__ __forceinline__ void cp_async8(float2* dst, const float2* src, bool valid)
{
	const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
	asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(valid ? 8 : 0) : "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait_n() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }
} // namespace

__global__ void k_pgr_phase(const PgrArgs p, int nb)
{
	const int a = blockIdx.x / nb, g = blockIdx.z;
	const int i = (blockIdx.x - a * nb) * blockDim.x + threadIdx.x;
	if (i >= p.nx + p.ny) return;
	const double2 fp = p.site_pos[(long long)g * p.nsite + p.atom_site[a]];
	if (i < p.nx) {
		p.tx[((long long)g * p.natom + a) * p.nx + i] = cis_turns_neg(fp.x * (double)freq(i, p.nx));
	}
	else {
		const int j = i - p.nx;
		const float2 e = cis_turns_neg(fp.y * (double)freq(j, p.ny));
		const float o = p.atom_occ[a];
		p.ty[((long long)g * p.natom + a) * p.ny + j] = make_float2(o * e.x, o * e.y);
	}
}

cudaError_t launch_pgr_phase(const PgrArgs& p, cudaStream_t s)
{
	if (p.natom <= 0 || p.ngr <= 0) return cudaSuccess;
	const int nb = (p.nx + p.ny + 255) / 256;
	k_pgr_phase<<<dim3((unsigned)(nb * p.natom), 1, p.ngr), 256, 0, s>>>(p, nb);
	return cudaGetLastError();
}

__global__ void k_pgr_fq(const PgrArgs p, float2* fq)
{
	const int ix = blockIdx.x * blockDim.x + threadIdx.x, iy = blockIdx.y, t = blockIdx.z;
	if (ix >= p.nx) return;
	const float qx = (float)freq(ix, p.nx) * p.itogx;
	const float qy = (float)freq(iy, p.ny) * p.itogy;
	const float q = sqrtf(__fadd_rn(__fmul_rn(qx, qx), __fmul_rn(qy, qy)));
	const float fpq = q / p.sk;
	int i0 = (int)fpq;
	i0 = min(i0, p.nk - 2);
	const float w1 = fpq - (float)i0;
	const float2* ff = p.ff + (long long)t * p.nk;
	const float2 f0 = __ldg(ff + i0), f1 = __ldg(ff + i0 + 1);
	float fr = f0.x * (1.f - w1) + f1.x * w1;
	float fi = f0.y * (1.f - w1) + f1.y * w1;
	if (p.bwl_pot) {
		const float ap = 0.5f - 0.5f * tanhf((q / p.kmax - 0.9f) * 30.f);
		fr *= ap * ap;
		fi *= ap * ap;
	}
	fq[((long long)t * p.ny + iy) * p.nx + ix] = make_float2(fr, fi);
}

cudaError_t launch_pgr_fq(const PgrArgs& p, float2* fq, cudaStream_t s)
{
	k_pgr_fq<<<dim3((p.nx + 255) / 256, p.ny, p.ntype), 256, 0, s>>>(p, fq);
	return cudaGetLastError();
}

// Chunks of 16 consecutive atoms (type order, across type boundaries) are
// staged by cp.async into one of two shared buffers while the previous chunk
// is summed; when a type's atoms end, f_t S_t and f_t conj(S_t) join the
// potentials at q and -q, which each thread keeps in 32 shared slots
// (registers hold only S).
__global__ void __launch_bounds__(kSThr, 2) k_pgr_synth(const PgrArgs p)
{
	extern __shared__ __align__(16) float2 smem[];     // 2 x kChunkF2 staging, then pot [32][kSThr]
	float2* pot = smem + 2 * kChunkF2 + threadIdx.x;   // slot k (q) and 16 + k (-q) at pot[slot * kSThr]
	const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5, g = blockIdx.z;
	const int hb = (p.ny + 1) >> 1;                    // rows summed here: iy < hb
	const int ix0 = blockIdx.x * kSX + 2 * lane;
	const int iy0 = blockIdx.y * kSY + kRW * wp;
	const float2* txg = p.tx + (long long)g * p.natom * p.nx;
	const float2* tyg = p.ty + (long long)g * p.natom * p.ny;
	const int natom = p.natom;
	const int nch = (natom + kCH - 1) / kCH;
	// staging: thread k copies table column / row r = k mod 128 of atoms
	// 2 m + k / 128 of a chunk (m < kCH / 2); ex [kCH][kSX] then ey [kCH][kSY]
	static_assert(kSX == kSY && kSThr == 2 * (kSX + kSY), "staging map");
	const int sr = threadIdx.x % (kSX + kSY), sa = threadIdx.x / (kSX + kSY);
	const bool sx = sr < kSX;
	const int sij = sx ? blockIdx.x * kSX + sr : blockIdx.y * kSY + sr - kSX;
	const bool sin = sx ? sij < p.nx : sij < hb;
	const float2* ssrc = (sx ? txg : tyg) + (sin ? sij : 0);
	const int sstr = sx ? p.nx : p.ny;
	const int sdst = (sx ? sr : kCH * kSX + sr - kSX) + sa * kSX;
	auto stage = [&](int c) {
		float2* buf = smem + (c & 1) * kChunkF2 + sdst;
		#pragma unroll
		for (int m = 0; m < kCH / 2; m++) {
			const int at = c * kCH + sa + 2 * m;
			const bool ok = sin && at < natom;
			cp_async8(buf + 2 * m * kSX, ok ? ssrc + (long long)at * sstr : ssrc, ok);
		}
		cp_async_commit();
	};
	float2 S[kRW][2];
	#pragma unroll
	for (int r = 0; r < kRW; r++) {
		S[r][0] = S[r][1] = make_float2(0.f, 0.f);
		#pragma unroll
		for (int c = 0; c < 2; c++) pot[(2 * r + c) * kSThr] = pot[(16 + 2 * r + c) * kSThr] = make_float2(0.f, 0.f);
	}
	// pot(q) += f_t S_t(q), pot(-q) += f_t conj(S_t(q)); S = 0
	auto close_type = [&](int t) {
		const float2* F = p.fq + (long long)t * p.nx * p.ny;
		#pragma unroll
		for (int r = 0; r < kRW; r++) {
			const int iy = iy0 + r;
			#pragma unroll
			for (int c = 0; c < 2; c++) {
				const int ix = ix0 + c;
				const float2 f = (ix < p.nx && iy < hb) ? __ldg(F + (long long)iy * p.nx + ix) : make_float2(0.f, 0.f);
				const float fr = f.x, fi = f.y;
				const float sxv = S[r][c].x, syv = S[r][c].y;
				float2 pv = pot[(2 * r + c) * kSThr];
				pv.x += fr * sxv - fi * syv;
				pv.y += fr * syv + fi * sxv;
				pot[(2 * r + c) * kSThr] = pv;
				float2 pm = pot[(16 + 2 * r + c) * kSThr];
				pm.x += fr * sxv - fi * (-syv);
				pm.y += fr * (-syv) + fi * sxv;
				pot[(16 + 2 * r + c) * kSThr] = pm;
				S[r][c] = make_float2(0.f, 0.f);
			}
		}
	};
	int t = 0, tend = p.type_start[1];
	while (t < p.ntype && tend == 0) { close_type(t); t++; if (t < p.ntype) tend = p.type_start[t + 1]; }
	if (nch > 0) stage(0);
	for (int c = 0; c < nch; c++) {
		if (c + 1 < nch) {
			stage(c + 1);
			cp_async_wait_n<1>();
		}
		else {
			cp_async_wait_n<0>();
		}
		__syncthreads();
		const float2* buf = smem + (c & 1) * kChunkF2;
		const int a0 = c * kCH, a1 = min(natom, a0 + kCH);
		int a = a0;
		while (a < a1) {
			const int aend = min(a1, tend);
			const float4* pe = reinterpret_cast<const float4*>(buf) + lane + (a - a0) * (kSX / 2);
			const float4* pw = reinterpret_cast<const float4*>(buf + kCH * kSX) + (kRW / 2) * wp + (a - a0) * (kSY / 2);
			#pragma unroll 2
			for (int n = aend - a; n > 0; n--, pe += kSX / 2, pw += kSY / 2) {
				const float4 e = *pe;                     // columns 2 lane, 2 lane + 1
				#pragma unroll
				for (int rr = 0; rr < kRW / 2; rr++) {
					const float4 w = pw[rr];              // rows 2 rr, 2 rr + 1 (broadcast)
					cmac(S[2 * rr][0], e.x, e.y, w.x, w.y);
					cmac(S[2 * rr][1], e.z, e.w, w.x, w.y);
					cmac(S[2 * rr + 1][0], e.x, e.y, w.z, w.w);
					cmac(S[2 * rr + 1][1], e.z, e.w, w.z, w.w);
				}
			}
			a = aend;
			// types whose atoms end here (and empty types after them)
			while (t < p.ntype && a == tend) {
				close_type(t);
				t++;
				if (t < p.ntype) tend = p.type_start[t + 1];
			}
		}
		__syncthreads();   // the buffer of chunk c is restaged for chunk c + 2
	}
	float2* out = p.out + (long long)g * p.gstride;
	const int nyqx = (p.nx & 1) ? -1 : (p.nx >> 1);    // column without a sampled mirror
	#pragma unroll
	for (int r = 0; r < kRW; r++) {
		const int iy = iy0 + r;
		if (iy >= hb) break;
		float2* o = out + (long long)iy * p.nx + ix0;
		const float2 v0 = pot[(2 * r) * kSThr], v1 = pot[(2 * r + 1) * kSThr];
		if (ix0 + 1 < p.nx && (p.nx & 1) == 0)
			*reinterpret_cast<float4*>(o) = make_float4(v0.x, v0.y, v1.x, v1.y);
		else {
			if (ix0 < p.nx) o[0] = v0;
			if (ix0 + 1 < p.nx) o[1] = v1;
		}
		if (iy == 0) continue;                          // row 0 is its own mirror: summed in full
		float2* om = out + (long long)(p.ny - iy) * p.nx;
		#pragma unroll
		for (int c = 0; c < 2; c++) {
			const int ix = ix0 + c;
			if (ix < p.nx && ix != nyqx) om[ix == 0 ? 0 : p.nx - ix] = pot[(16 + 2 * r + c) * kSThr];
		}
	}
}

// The pixels without a sampled mirror: the Nyquist row ny / 2 (even ny, all
// columns), then the Nyquist column nx / 2 (even nx) of the mirrored rows
// ny - iy, 1 <= iy < ceil(ny / 2).  A CTA takes 32 consecutive pixels (one
// per lane, so the table reads coalesce); its 8 warps share the atoms of each
// type (warp w: atoms w, w + 8, ...), and warp 0 adds their partial sums in
// warp order.
constexpr int kLineWarps = 8;
__global__ void __launch_bounds__(32 * kLineWarps) k_pgr_lines(const PgrArgs p, int nrow, int npts)
{
	__shared__ float2 part[kLineWarps][32];
	const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, g = blockIdx.z;
	const int k = blockIdx.x * 32 + lane;
	const bool live = k < npts;
	int ix = 0, iy = 0;
	if (k < nrow) { ix = k; iy = p.ny >> 1; }
	else if (live) { ix = p.nx >> 1; iy = p.ny - (1 + k - nrow); }
	const float2* txg = p.tx + (long long)g * p.natom * p.nx + ix;
	const float2* tyg = p.ty + (long long)g * p.natom * p.ny + iy;
	float2 pot = make_float2(0.f, 0.f);
	for (int t = 0; t < p.ntype; t++) {
		float2 S = make_float2(0.f, 0.f);
		if (live)
			for (int a = p.type_start[t] + w; a < p.type_start[t + 1]; a += kLineWarps) {
				const float2 e = __ldg(txg + (long long)a * p.nx), v = __ldg(tyg + (long long)a * p.ny);
				cmac(S, e.x, e.y, v.x, v.y);
			}
		part[w][lane] = S;
		__syncthreads();
		if (w == 0 && live) {
			S = part[0][lane];
			#pragma unroll
			for (int q = 1; q < kLineWarps; q++) S = make_float2(S.x + part[q][lane].x, S.y + part[q][lane].y);
			const float2 f = __ldg(p.fq + ((long long)t * p.ny + iy) * p.nx + ix);
			const float fr = f.x, fi = f.y;
			pot.x += fr * S.x - fi * S.y;
			pot.y += fr * S.y + fi * S.x;
		}
		__syncthreads();
	}
	if (w == 0 && live) p.out[(long long)g * p.gstride + (long long)iy * p.nx + ix] = pot;
}

cudaError_t launch_pgr_synth(const PgrArgs& p, cudaStream_t s)
{
	constexpr int smem = (2 * kChunkF2 + 32 * kSThr) * (int)sizeof(float2);
	// the dynamic shared-memory limit is raised once per device
	static bool attr_set[64] = {};
	int dev = 0;
	cudaError_t e = cudaGetDevice(&dev);
	if (e != cudaSuccess) return e;
	if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
	if (!attr_set[dev]) {
		e = cudaFuncSetAttribute(k_pgr_synth, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
		if (e != cudaSuccess) return e;
		attr_set[dev] = true;
	}
	const int hb = (p.ny + 1) >> 1;
	const dim3 grid((p.nx + kSX - 1) / kSX, (hb + kSY - 1) / kSY, p.ngr);
	k_pgr_synth<<<grid, kSThr, smem, s>>>(p);
	if ((e = cudaGetLastError()) != cudaSuccess) return e;
	// pixels without a sampled mirror: Nyquist row (even ny), Nyquist column
	// of the mirrored rows (even nx)
	const int nrow = (p.ny & 1) ? 0 : p.nx;
	const int ncol = (p.nx & 1) ? 0 : hb - 1;
	const int npts = nrow + ncol;
	if (npts > 0) {
		k_pgr_lines<<<dim3((npts + 31) / 32, 1, p.ngr), 32 * kLineWarps, 0, s>>>(p, nrow, npts);
		e = cudaGetLastError();
	}
	return e;
}

// ---------------------------------------------------------------------------
// line transforms of the generator (default line plan of each length)
// ---------------------------------------------------------------------------
namespace {
const PgrOps* pgr_ops(int n)
{
	if (const PgrOps* o = pgr_ops_0(n)) return o;
	if (const PgrOps* o = pgr_ops_1(n)) return o;
	return pgr_ops_2(n);
}
} // namespace

bool pgr_supported(int nx, int ny) { return pgr_ops(nx) && pgr_ops(ny); }

cudaError_t launch_pgr_rows_inv(const PgrArgs& p, cudaStream_t s)
{
	const PgrOps* o = pgr_ops(p.nx);
	return o ? o->rows_inv(p, s) : cudaErrorInvalidValue;
}

cudaError_t launch_pgr_cols(const PgrArgs& p, const float2* src, float2* dst, int mode, cudaStream_t s)
{
	const PgrOps* o = pgr_ops(p.ny);
	return o ? o->cols(p, src, dst, mode, s) : cudaErrorInvalidValue;
}

} // namespace jms
