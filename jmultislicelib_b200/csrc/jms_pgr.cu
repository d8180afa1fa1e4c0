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
// A CTA owns a 32 x 32 pixel tile of one grating: thread (x = lane, group)
// accumulates 4 rows of one column.  The translation phase is separable,
// exp(-2 pi i (x qx + y qy)) = ex(qx) ey(qy); per chunk of 32 atoms the CTA
// tabulates ex for its 32 columns and occ * ey for its 32 rows in shared
// memory (64 sincos per atom instead of 1024), the phase in turns x/a * fi
// formed in FP64 and reduced to [-1/2, 1/2) before the FP32 sincospi.
namespace {
constexpr int kSX = 32, kSG = 8, kSR = 4, kSY = kSG * kSR, kCH = 32;

__device__ __forceinline__ int freq(int i, int n)
{
	const int h = (n - (n % 2)) >> 1;
	return ((i + h) % n) - h;
}

__device__ __forceinline__ float2 cis_turns_neg(double t)
{
	t -= rint(t);
	float s, c;
	sincospif(2.f * (float)t, &s, &c);
	return make_float2(c, -s);
}
} // namespace

__global__ void __launch_bounds__(kSX * kSG) k_pgr_synth(const PgrArgs p)
{
	__shared__ float2 ex[kCH][kSX];
	__shared__ float2 ey[kCH][kSY];
	const int lane = threadIdx.x & 31, grp = threadIdx.x >> 5, g = blockIdx.z;
	const int ix = blockIdx.x * kSX + lane;
	const int iy0 = blockIdx.y * kSY;
	const double2* pos = p.site_pos + (long long)g * p.nsite;
	const float qx = (float)freq(ix < p.nx ? ix : 0, p.nx) * p.itogx;
	float2 pot[kSR];
	#pragma unroll
	for (int r = 0; r < kSR; r++) pot[r] = make_float2(0.f, 0.f);
	for (int t = 0; t < p.ntype; t++) {
		float2 S[kSR];
		#pragma unroll
		for (int r = 0; r < kSR; r++) S[r] = make_float2(0.f, 0.f);
		const int a0 = p.type_start[t], a1 = p.type_start[t + 1];
		for (int c0 = a0; c0 < a1; c0 += kCH) {
			const int na = min(kCH, a1 - c0);
			__syncthreads();
			for (int k = threadIdx.x; k < na * (kSX + kSY); k += kSX * kSG) {
				const int a = k / (kSX + kSY), r = k % (kSX + kSY);
				const int at = c0 + a;
				const double2 fp = pos[p.atom_site[at]];
				if (r < kSX) {
					const int i = blockIdx.x * kSX + r;
					ex[a][r] = cis_turns_neg(fp.x * (double)freq(i < p.nx ? i : 0, p.nx));
				}
				else {
					const int j = iy0 + r - kSX;
					const float2 e = cis_turns_neg(fp.y * (double)freq(j < p.ny ? j : 0, p.ny));
					const float o = p.atom_occ[at];
					ey[a][r - kSX] = make_float2(o * e.x, o * e.y);
				}
			}
			__syncthreads();
			for (int a = 0; a < na; a++) {
				const float2 e = ex[a][lane];
				#pragma unroll
				for (int r = 0; r < kSR; r++) {
					const float2 w = ey[a][grp * kSR + r];     // broadcast
					S[r].x = fmaf(e.x, w.x, fmaf(-e.y, w.y, S[r].x));
					S[r].y = fmaf(e.x, w.y, fmaf(e.y, w.x, S[r].y));
				}
			}
		}
		// pot += f_t(|q|) ap1(q)^2 S_t(q)
		const float2* ff = p.ff + (long long)t * p.nk;
		#pragma unroll
		for (int r = 0; r < kSR; r++) {
			const int iy = iy0 + grp * kSR + r;
			const float qy = (float)freq(iy < p.ny ? iy : 0, p.ny) * p.itogy;
			const float q = sqrtf(__fadd_rn(__fmul_rn(qx, qx), __fmul_rn(qy, qy)));
			const float fpq = q / p.sk;
			int i0 = (int)fpq;
			i0 = min(i0, p.nk - 2);
			const float w1 = fpq - (float)i0;
			const float2 f0 = __ldg(ff + i0), f1 = __ldg(ff + i0 + 1);
			float fr = f0.x * (1.f - w1) + f1.x * w1;
			float fi = f0.y * (1.f - w1) + f1.y * w1;
			if (p.bwl_pot) {
				const float ap = 0.5f - 0.5f * tanhf((q / p.kmax - 0.9f) * 30.f);
				fr *= ap * ap;
				fi *= ap * ap;
			}
			pot[r].x += fr * S[r].x - fi * S[r].y;
			pot[r].y += fr * S[r].y + fi * S[r].x;
		}
	}
	if (ix >= p.nx) return;
	float2* out = p.out + (long long)g * p.gstride;
	#pragma unroll
	for (int r = 0; r < kSR; r++) {
		const int iy = iy0 + grp * kSR + r;
		if (iy < p.ny) out[(long long)iy * p.nx + ix] = pot[r];
	}
}

cudaError_t launch_pgr_synth(const PgrArgs& p, cudaStream_t s)
{
	const dim3 grid((p.nx + kSX - 1) / kSX, (p.ny + kSY - 1) / kSY, p.ngr);
	k_pgr_synth<<<grid, kSX * kSG, 0, s>>>(p);
	return cudaGetLastError();
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
