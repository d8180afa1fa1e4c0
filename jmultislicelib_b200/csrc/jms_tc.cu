// jms_tc.cu -- tensor-core (tcgen05) forms of the fused multislice passes.
//
// Same passes as the FP32 kernels of jms_passes.cuh (row pass FT_x -> x P ->
// IFT_x, column pass IFT_y -> x t -> FT_y; reference slice loop
// src/JMultiSlice.cpp:4590-4651, unnormalised transforms as
// src/JFFTCUDAcore.cpp:299-336), with every radix stage of the line
// transforms run as a small dense DFT-matrix product on the tensor cores.
//
// Line transform.  A line of N = R1 * R2 points (x[R2 n1 + n2]) is
// transformed in two radix stages:
//   stage 1: Y[n2][k1] = sum_n1 x[R2 n1 + n2] W_R1^(n1 k1), times W_N^(n2 k1)
//   stage 2: X[k1 + R1 k2] = sum_n2 Y[n2][k1] W_R2^(n2 k2)
// and the inverse through conj(F(conj(.))).  A stage over a batch of rows
// (one row = the R values a radix-R DFT contracts) is D = A B^T with
//   A  = rows x 2R real operand (re, im interleaved), in shared memory;
//   B  = the real-ified R-point DFT matrix (2R x 2R), in shared memory;
//   D  = rows x 2R FP32 accumulator in tensor memory (128 lanes = 128 rows).
// Precision: the wave operand A is split into 16-bit hi + lo parts (BF16 or
// FP16), the constant DFT matrix B into hi + mid + lo, and
//   D = A_hi B_hi + (A_lo B_hi + A_hi B_mid + A_lo B_mid + A_hi B_lo)
// with FP32 accumulation: the main product A_hi B_hi in one TMEM accumulator,
// the four correction products (2^-8 / 2^-9 of it) in a second one, added in
// FP32 registers after the MMAs.  Each MMA step that adds into an accumulator
// rounds at that accumulator's magnitude, and that rounding is biased (it
// added up coherently from slice to slice in the measurements), so only the
// K / 16 steps of the main product run at the magnitude of the result, and
// that product is kept 16 bits wide (8-bit hi parts) so its sums lose (almost)
// nothing.  The matrix carries no error of its own (8 + 11 + 11 / 3 x 8
// bits); the unbiased rounding of A to 19 (FP16, 8 + 11) / 16 (BF16)
// significant bits is what remains.
// FP16 operands carry a power-of-two scale per tile (max |value| -> 2^14),
// removed exactly after the MMA.
//
// Tile.  A CTA of 512 threads owns a tile of T = 4096 points: L = T / N
// lines of length N (rows of the wave in the row pass, adjacent columns in
// the column pass).  Its rows come in two sets:
//   P: (line l, n2), R1 values each (stage-1 rows), T / R1 rows;
//   Q: (line l, k1), R2 values each (stage-2 rows), T / R2 rows;
// 4 threads serve each TMEM lane: thread t owns rows t % 128 + 128 j of the
// current set, holds the quarter t / 128 of their values (8 complex values
// per thread, 64 registers) and reads that quarter of their D rows from its
// lane.  Between the two stages a thread writes its values into the other
// set's A operand (the transpose of the FFT), through layouts padded so that
// those writes are free of bank conflicts.  The elementwise step of the pass
// (x P, or x t) runs in registers between the halves, so a line is read from
// and written to HBM once per pass, as in the FP32 kernels.  The kernels are
// persistent: a CTA copies the DFT matrices (built once per device) and
// builds its twiddles in shared memory, then walks its tiles, loading the
// next tile's input while the MMAs of the current tile's last stage run.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include "jms_fft.cuh"
#include "jms_kernels.h"
#include "jms_launch.cuh"
#include "jms_tc.cuh"

namespace jms {
namespace tc {

constexpr int kLanes = 128;           // rows of an MMA tile = TMEM lanes (M = 128)
constexpr int kQ = 4;                 // threads per TMEM lane: each holds a quarter of its rows' values
constexpr int kThr = kLanes * kQ;     // threads per CTA
// complex points per tile: 4096, or 8192 for N = 2048 (4 lines, so that the
// 64-point stage's (line, n2) rows still fill M = 128)
__host__ __device__ constexpr int tile_of(int n) { return n == 2048 ? 8192 : 4096; }
constexpr long long kMaxWaitCycles = 2000000000LL; // ~1 s at 1.9 GHz, then the pass reports an error

template <int N> struct Radix;
template <> struct Radix<256> { static constexpr int R1 = 16, R2 = 16; };
template <> struct Radix<512> { static constexpr int R1 = 32, R2 = 16; };
template <> struct Radix<1024> { static constexpr int R1 = 32, R2 = 32; };
template <> struct Radix<2048> { static constexpr int R1 = 64, R2 = 32; };

// (LBO, SBO) of the A layouts of sets P and Q, chosen by a bank-conflict
// search over the transposing writes (conflict-free except the 256-point
// column passes of 256 and 2048 points, which are 2-way; the conflict-free
// 2048-point column layout would not fit in shared memory)
template <int N, bool COL> struct Lay;
template <> struct Lay<256, false> { static constexpr int lp = 144, sp = 608, lq = 144, sq = 608; };
template <> struct Lay<512, false> { static constexpr int lp = 144, sp = 1152, lq = 144, sq = 592; };
template <> struct Lay<1024, false> { static constexpr int lp = 144, sp = 1152, lq = 144, sq = 1152; };
template <> struct Lay<256, true> { static constexpr int lp = 128, sp = 512, lq = 128, sq = 512; };
template <> struct Lay<512, true> { static constexpr int lp = 128, sp = 1024, lq = 128, sq = 512; };
template <> struct Lay<1024, true> { static constexpr int lp = 192, sp = 1536, lq = 192, sq = 1536; };
template <> struct Lay<2048, false> { static constexpr int lp = 144, sp = 2304, lq = 144, sq = 1152; };
template <> struct Lay<2048, true> { static constexpr int lp = 128, sp = 2048, lq = 128, sq = 1024; };

constexpr int rup(int x, int a) { return (x + a - 1) / a * a; }
constexpr int cmax(int a, int b) { return a > b ? a : b; }

template <int N, bool COL>
struct Geo {
	static constexpr int R1 = Radix<N>::R1, R2 = Radix<N>::R2;
	static constexpr int T = tile_of(N);                 // points per tile
	static constexpr int NV = T / kThr;                  // complex values per thread
	static constexpr int DC = T / 64;                    // FP32 accumulator columns of a stage (J 2R = 2 T / 128)
	static constexpr int TCOLS = 2 * DC;                 // main + correction accumulators
	static constexpr int L = T / N;                      // lines per tile
	static constexpr int MP = L * R2, MQ = L * R1;       // rows of sets P and Q
	static constexpr int JP = MP / kLanes, JQ = MQ / kLanes; // rows per TMEM lane (and per thread)
	static constexpr int VP = R1 / kQ, VQ = R2 / kQ;         // values per thread and row in P / Q
	static constexpr int LP = Lay<N, COL>::lp, SP = Lay<N, COL>::sp, LQ = Lay<N, COL>::lq, SQ = Lay<N, COL>::sq;
	static_assert(MP % kLanes == 0 && MQ % kLanes == 0, "tile rows must fill M = 128");
	static_assert(VP % 4 == 0 && VQ % 4 == 0, "a thread writes whole 16-byte chunks of its rows");
	static_assert(SP >= (R1 / 4) * LP && SQ >= (R2 / 4) * LQ, "layout rows overlap");
	static constexpr int bytes(int M, int KC, int lbo, int sbo) { return (M / 8 - 1) * sbo + (KC - 1) * lbo + 128; }
	static constexpr int kA = rup(cmax(bytes(MP, R1 / 4, LP, SP), bytes(MQ, R2 / 4, LQ, SQ)), 1024);
	static constexpr int kF1 = 8 * R1 * R1, kF2 = (R2 == R1) ? 0 : 8 * R2 * R2; // bytes of one matrix term
	static constexpr int TWS = R2 + 1;                   // padded row of the twiddle table W[k1][n2]
	// offsets: A_hi, A_lo, F1 (hi, mid, lo), F2 (hi, mid, lo), W[k1][n2]
	static constexpr int oAlo = kA, oF1 = 2 * kA, oF2 = oF1 + 3 * kF1, oW = oF2 + 3 * kF2;
	static constexpr int kSmem = oW + R1 * TWS * 8;
	__device__ static int prow(int l, int n2) { return COL ? n2 * L + l : l * R2 + n2; }
	__device__ static int qrow(int l, int k1) { return COL ? k1 * L + l : l * R1 + k1; }
	// byte offset of row m in a layout with row-group stride SB, split into a
	// part from the line l (runtime) and a part from the digit (compile-time
	// in the unrolled loops): off(row(l, d)) = lbase(l) + dconst(d)
	template <int SB, int D>
	__device__ static int lbase(int l)
	{
		if (COL) return L >= 8 ? (l >> 3) * SB + (l & 7) * 16 : l * 16;   // l < L
		return l * (D / 8) * SB;                                           // D = digits per line (8 | D)
	}
	template <int SB>
	__device__ static constexpr int dconst(int d)
	{
		if (COL) return L >= 8 ? d * (L / 8) * SB : ((d * L) >> 3) * SB + ((d * L) & 7) * 16;
		return (d >> 3) * SB + (d & 7) * 16;
	}
	__device__ static void pinv(int m, int& l, int& n2)
	{
		if (COL) { l = m % L; n2 = m / L; }
		else { l = m / R2; n2 = m % R2; }
	}
	__device__ static void qinv(int m, int& l, int& k1)
	{
		if (COL) { l = m % L; k1 = m / L; }
		else { l = m / R1; k1 = m % R1; }
	}
};

// 16-bit operand types: split of FP32 values into hi + lo (round to nearest;
// a - hi is exact in FP32)
struct Bf16 {
	static constexpr uint32_t kFmt = 1;
	static constexpr bool kScale = false;
	__device__ static void split2(float a, float b, uint32_t& hi, uint32_t& lo)
	{
		const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
		const float2 hf = __bfloat1622float2(h);
		const __nv_bfloat162 l = __floats2bfloat162_rn(a - hf.x, b - hf.y);
		hi = *reinterpret_cast<const uint32_t*>(&h);
		lo = *reinterpret_cast<const uint32_t*>(&l);
	}
	__device__ static float round1(float a, uint16_t& bits)
	{
		const __nv_bfloat16 h = __float2bfloat16_rn(a);
		bits = *reinterpret_cast<const uint16_t*>(&h);
		return __bfloat162float(h);
	}
	__device__ static float round_hi(float a, uint16_t& bits) { return round1(a, bits); }
};
// FP16: the hi part is rounded to 8 significant bits (through BF16; exact in
// FP16 within the scaled range) and the lo part keeps 11 more, so A is held to
// 2^-21 while hi x hi products stay 16-bit wide: their sums in the main
// accumulator then lose (almost) nothing to the accumulation's rounding.
struct Fp16 {
	static constexpr uint32_t kFmt = 0;
	static constexpr bool kScale = true;
	__device__ static void split2(float a, float b, uint32_t& hi, uint32_t& lo)
	{
		const float2 hf = __bfloat1622float2(__floats2bfloat162_rn(a, b));
		const __half2 h = __floats2half2_rn(hf.x, hf.y);
		const __half2 l = __floats2half2_rn(a - hf.x, b - hf.y);
		hi = *reinterpret_cast<const uint32_t*>(&h);
		lo = *reinterpret_cast<const uint32_t*>(&l);
	}
	__device__ static float round1(float a, uint16_t& bits)
	{
		const __half h = __float2half_rn(a);
		bits = *reinterpret_cast<const uint16_t*>(&h);
		return __half2float(h);
	}
	// first term of a constant: 8 significant bits, as the operand's hi part
	__device__ static float round_hi(float a, uint16_t& bits)
	{
		const __half h = __float2half_rn(__bfloat162float(__float2bfloat16_rn(a)));
		bits = *reinterpret_cast<const uint16_t*>(&h);
		return __half2float(h);
	}
};

__device__ __forceinline__ float2 conjf2(float2 a) { return make_float2(a.x, -a.y); }
__device__ __forceinline__ int opaque(int x)
{
	int y;
	asm volatile("mov.b32 %0, %1;" : "=r"(y) : "r"(x));
	return y;
}

// Real-ified R-point forward DFT matrix as the B operand (2R x 2R, K-major,
// LBO 128, SBO 32 R), in three 16-bit terms hi + mid + lo at f, f + 8R^2,
// f + 16R^2: row 2k + c (output k, re / im), column 2q + d (input q, re /
// im).  cos and sin of 2 pi (kq mod R) / R are computed in FP64 and split
// from there, so hi + mid + lo holds them to 2^-30 (FP16) / 2^-24 (BF16).
template <int R, class PR>
__device__ void build_dft(uint8_t* f)
{
	for (int e = threadIdx.x; e < 4 * R * R; e += kThr) {
		const int nout = e / (2 * R), kin = e % (2 * R);
		const int k = nout >> 1, c = nout & 1, q = kin >> 1, d = kin & 1;
		double sn, cs;
		sincospi(2.0 * (double)((k * q) % R) / (double)R, &sn, &cs);
		const double val = (c == 0) ? (d == 0 ? cs : sn) : (d == 0 ? -sn : cs);
		uint16_t bh, bm, bl;
		const double h = (double)PR::round_hi((float)val, bh);
		const double m = (double)PR::round1((float)(val - h), bm);
		PR::round1((float)(val - h - m), bl);
		const int off = (nout >> 3) * (32 * R) + (kin >> 3) * 128 + (nout & 7) * 16 + (kin & 7) * 2;
		*reinterpret_cast<uint16_t*>(f + off) = bh;
		*reinterpret_cast<uint16_t*>(f + 8 * R * R + off) = bm;
		*reinterpret_cast<uint16_t*>(f + 16 * R * R + off) = bl;
	}
}

// DFT matrices of both radices and operand types, built once per device by
// k_build_dft (tc_prepare) and copied into shared memory by each CTA:
// [type (0 BF16, 1 FP16)][R = 16 (6144 B), R = 32 (24576 B)]
constexpr int kDftType = 3 * 8 * (16 * 16 + 32 * 32 + 64 * 64);
__device__ __align__(16) uint8_t g_dft[2 * kDftType];
__host__ __device__ constexpr int dft_off(int type, int R)
{
	return type * kDftType + (R == 16 ? 0 : R == 32 ? 3 * 8 * 16 * 16 : 3 * 8 * (16 * 16 + 32 * 32));
}

__global__ void __launch_bounds__(kThr) k_build_dft()
{
	switch (blockIdx.x) {
	case 0: build_dft<16, Bf16>(g_dft + dft_off(0, 16)); break;
	case 1: build_dft<32, Bf16>(g_dft + dft_off(0, 32)); break;
	case 2: build_dft<64, Bf16>(g_dft + dft_off(0, 64)); break;
	case 3: build_dft<16, Fp16>(g_dft + dft_off(1, 16)); break;
	case 4: build_dft<32, Fp16>(g_dft + dft_off(1, 32)); break;
	default: build_dft<64, Fp16>(g_dft + dft_off(1, 64)); break;
	}
}

template <int R>
__device__ __forceinline__ void copy_dft(uint8_t* dst, int type)
{
	const uint4* src = reinterpret_cast<const uint4*>(g_dft + dft_off(type, R));
	for (int i = threadIdx.x; i < 3 * 8 * R * R / 16; i += kThr) reinterpret_cast<uint4*>(dst)[i] = src[i];
}

// Per-tile power-of-two operand scale (FP16 only): returns s with
// max |v| * s < 2^14; *inv = 1 / s.  Block-wide (every thread calls it).
template <class PR, int NV>
__device__ __forceinline__ float tile_scale(const float2 (&v)[NV], float* red, float* inv)
{
	if constexpr (!PR::kScale) {
		*inv = 1.f;
		return 1.f;
	}
	else {
		float mx = 0.f;
		#pragma unroll
		for (int q = 0; q < NV; q++) mx = fmaxf(mx, fmaxf(fabsf(v[q].x), fabsf(v[q].y)));
		#pragma unroll
		for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
		if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
		__syncthreads();
		mx = 0.f;
		#pragma unroll
		for (int w = 0; w < kThr / 32; w++) mx = fmaxf(mx, red[w]);
		int e = 0;
		if (mx > 0.f) frexpf(mx, &e);
		e = max(min(e, 100), -100);
		*inv = ldexpf(1.f, e - 14);
		return ldexpf(1.f, 14 - e);
	}
}

// Thread t serves TMEM lane t % 128 (rows t % 128 + 128 j of the current
// set) and quarter q = t / 128 of those rows' values: value index q V + i,
// i < V = R / 4, held in v[j V + i].
__device__ __forceinline__ int lane_of() { return threadIdx.x & (kLanes - 1); }
__device__ __forceinline__ int quarter_of() { return threadIdx.x >> 7; }

// A operand of a set whose rows are the thread's own rows: row m, 16-byte
// chunk c = values 4c .. 4c+3 (8 16-bit numbers); the thread writes the
// chunks of its quarter
template <int R, int J, int LB, int SB, class PR, int NV>
__device__ __forceinline__ void write_own(const float2 (&v)[NV], uint8_t* ahi, uint8_t* alo, float s)
{
	constexpr int V = R / kQ;
	#pragma unroll
	for (int j = 0; j < J; j++) {
		const int m = lane_of() + kLanes * j;
		const int base = (m >> 3) * SB + (m & 7) * 16 + quarter_of() * (V / 4) * LB;
		#pragma unroll
		for (int c = 0; c < V / 4; c++) {
			uint4 h, l;
			PR::split2(v[j * V + 4 * c + 0].x * s, v[j * V + 4 * c + 0].y * s, h.x, l.x);
			PR::split2(v[j * V + 4 * c + 1].x * s, v[j * V + 4 * c + 1].y * s, h.y, l.y);
			PR::split2(v[j * V + 4 * c + 2].x * s, v[j * V + 4 * c + 2].y * s, h.z, l.z);
			PR::split2(v[j * V + 4 * c + 3].x * s, v[j * V + 4 * c + 3].y * s, h.w, l.w);
			*reinterpret_cast<uint4*>(ahi + base + c * LB) = h;
			*reinterpret_cast<uint4*>(alo + base + c * LB) = l;
		}
	}
}

// transposing write P -> Q: the thread's P rows (l, n2) hold values over k1
// (its quarter); Q row (l, k1) gets value n2 at K position n2
template <class G, class PR, int NV>
__device__ __forceinline__ void write_pq(const float2 (&v)[NV], uint8_t* ahi, uint8_t* alo, float s)
{
	constexpr int V = G::VP;
	#pragma unroll
	for (int j = 0; j < G::JP; j++) {
		int l, n2;
		G::pinv(lane_of() + kLanes * j, l, n2);
		uint8_t* bh = ahi + G::template lbase<G::SQ, G::R1>(l) + (n2 >> 2) * G::LQ + (n2 & 3) * 4 +
			G::template dconst<G::SQ>(quarter_of() * V);
		uint8_t* bl = bh + (alo - ahi);
		#pragma unroll
		for (int i = 0; i < V; i++) {
			const int off = G::template dconst<G::SQ>(i);   // k1 = q V + i
			uint32_t h, lo;
			PR::split2(v[j * V + i].x * s, v[j * V + i].y * s, h, lo);
			*reinterpret_cast<uint32_t*>(bh + off) = h;
			*reinterpret_cast<uint32_t*>(bl + off) = lo;
		}
	}
}

// transposing write Q -> P: the thread's Q rows (l, k1) hold values over n2
// (its quarter); P row (l, n2) gets value k1 at K position k1
template <class G, class PR, int NV>
__device__ __forceinline__ void write_qp(const float2 (&v)[NV], uint8_t* ahi, uint8_t* alo, float s)
{
	constexpr int V = G::VQ;
	#pragma unroll
	for (int j = 0; j < G::JQ; j++) {
		int l, k1;
		G::qinv(lane_of() + kLanes * j, l, k1);
		uint8_t* bh = ahi + G::template lbase<G::SP, G::R2>(l) + (k1 >> 2) * G::LP + (k1 & 3) * 4 +
			G::template dconst<G::SP>(quarter_of() * V);
		uint8_t* bl = bh + (alo - ahi);
		#pragma unroll
		for (int i = 0; i < V; i++) {
			const int off = G::template dconst<G::SP>(i);   // n2 = q V + i
			uint32_t h, lo;
			PR::split2(v[j * V + i].x * s, v[j * V + i].y * s, h, lo);
			*reinterpret_cast<uint32_t*>(bh + off) = h;
			*reinterpret_cast<uint32_t*>(bl + off) = lo;
		}
	}
}

// V complex values (2V columns from taddr) of a D row: main accumulator +
// correction accumulator
template <int V, int DC>
__device__ __forceinline__ void tmem_ld_vals(uint32_t taddr, float2* dst, float inv)
{
	uint32_t r[2 * V], c[2 * V];
	if constexpr (V == 4) { tmem_ld8(taddr, r); tmem_ld8(taddr + DC, c); }
	else if constexpr (V == 8) { tmem_ld16(taddr, r); tmem_ld16(taddr + DC, c); }
	else { tmem_ld32(taddr, r); tmem_ld32(taddr + DC, c); }
	tmem_wait_ld();
	#pragma unroll
	for (int q = 0; q < V; q++)
		dst[q] = make_float2((__uint_as_float(r[2 * q]) + __uint_as_float(c[2 * q])) * inv,
			(__uint_as_float(r[2 * q + 1]) + __uint_as_float(c[2 * q + 1])) * inv);
}

// One radix stage over the current A operand, in three steps:
//   stage_issue: make the A writes visible to the tensor core, then thread 0
//                issues the MMAs and commits them to the mbarrier;
//   stage_wait:  thread 0 waits for them (bounded); the block learns the
//                outcome at a barrier whose ordering the tcgen05 fences extend
//                to the TMEM reads; false (uniformly) if they did not finish;
//   stage_read:  every thread reads its J rows of D (R complex each).
// Between issue and wait a thread may do work that does not touch A or D
// (the passes prefetch their next tile there).
template <int R, int J, int LB, int SB, class PR, int DC>
__device__ __forceinline__ void stage_issue(const uint8_t* ahi, const uint8_t* alo, const uint8_t* f, uint32_t tmem,
	uint32_t mbar)
{
	fence_async_smem();
	fence_before_sync();
	__syncthreads();
	if (threadIdx.x == 0) {
		fence_after_sync();
		constexpr uint32_t idesc = idesc_f16(PR::kFmt, kLanes, 2 * R);
		const uint32_t ah = smem_u32(ahi), al = smem_u32(alo), bh = smem_u32(f);
		const uint32_t bm = bh + 8 * R * R, bl = bh + 16 * R * R;
		#pragma unroll
		for (int i = 0; i < J; i++) {
			const uint32_t d = tmem + (uint32_t)(i * 2 * R);
			#pragma unroll
			for (int kk = 0; kk < 2 * R / 16; kk++) {
				const uint32_t ao = (uint32_t)(i * 16 * SB + kk * 2 * LB), bo = (uint32_t)(kk * 256);
				const uint64_t dah = sdesc(ah + ao, LB, SB), dal = sdesc(al + ao, LB, SB);
				const uint64_t dbh = sdesc(bh + bo, 128, 32 * R), dbm = sdesc(bm + bo, 128, 32 * R);
				const uint64_t dbl = sdesc(bl + bo, 128, 32 * R);
				const uint32_t acc = kk > 0 ? 1u : 0u;
				mma_f16(d, dah, dbh, idesc, acc);
				mma_f16(d + DC, dal, dbh, idesc, acc);
				mma_f16(d + DC, dah, dbm, idesc, 1u);
				mma_f16(d + DC, dal, dbm, idesc, 1u);
				mma_f16(d + DC, dah, dbl, idesc, 1u);
			}
		}
		mma_commit(mbar);
	}
}

__device__ __forceinline__ bool stage_wait(uint32_t mbar, uint32_t& phase)
{
	bool ok = true;
	if (threadIdx.x == 0) {
		ok = mbar_wait(mbar, phase, kMaxWaitCycles);
		fence_before_sync();
	}
	phase ^= 1u;
	if (__syncthreads_or(!ok)) return false;
	fence_after_sync();
	return true;
}

// TMEM address of the thread's lane quadrant (warp % 4) and quarter of a
// stage's D row (tile i, radix R): lane bits 31..16, column bits 15..0
template <int R>
__device__ __forceinline__ uint32_t d_addr(uint32_t tmem, int i)
{
	return tmem + ((uint32_t)(((threadIdx.x >> 5) & 3) * 32) << 16) + (uint32_t)(i * 2 * R + quarter_of() * 2 * (R / kQ));
}

template <int R, int J, int DC, int NV>
__device__ __forceinline__ void stage_read(float2 (&v)[NV], uint32_t tmem, float inv)
{
	#pragma unroll
	for (int i = 0; i < J; i++) tmem_ld_vals<R / kQ, DC>(d_addr<R>(tmem, i), &v[i * (R / kQ)], inv);
}

template <int R, int J, int LB, int SB, class PR, int DC, int NV>
__device__ __forceinline__ bool stage(float2 (&v)[NV], const uint8_t* ahi, const uint8_t* alo, const uint8_t* f,
	uint32_t tmem, uint32_t mbar, uint32_t& phase, float inv)
{
	stage_issue<R, J, LB, SB, PR, DC>(ahi, alo, f, tmem, mbar);
	if (!stage_wait(mbar, phase)) return false;
	stage_read<R, J, DC>(v, tmem, inv);
	return true;
}

struct TcTiles {
	long long ntiles = 0;
	int per_wave = 0;          // tiles per wave
	int split = 0, skip = 0;   // row pass: live row blocks [0, split) and [split + skip, nrb)
	int* err = nullptr;        // set to 1 if an MMA wait ran out
};

template <int N, bool COL, class PR>
__global__ void __launch_bounds__(kThr, N == 2048 ? 1 : 2) k_tc_pass(const PassArgs p, const TcTiles tt)
{
	using G = Geo<N, COL>;
	constexpr int R1 = G::R1, R2 = G::R2, L = G::L, VP = G::VP, VQ = G::VQ, DC = G::DC;
	extern __shared__ __align__(1024) uint8_t sm[];
	__shared__ __align__(8) uint64_t mbar_s;
	__shared__ uint32_t tbase_s;
	__shared__ float red_s[kThr / 32];
	uint8_t* ahi = sm;
	uint8_t* alo = sm + G::oAlo;
	const uint8_t* f1 = sm + G::oF1;
	const uint8_t* f2 = (R2 == R1) ? f1 : sm + G::oF2;
	// W_N^(n2 k1) at [k1][n2] with rows padded to R2 + 1: lanes of consecutive
	// n2 (same k1) and of consecutive k1 (same n2) both read without conflicts
	float2* wt = reinterpret_cast<float2*>(sm + G::oW);
	constexpr int TWS = G::TWS;
	const int tid = threadIdx.x;
	const int lane = lane_of(), q = quarter_of();
	const float2* tw = COL ? p.twy : p.twx;

	copy_dft<R1>(sm + G::oF1, PR::kFmt == 1 ? 0 : 1);
	if (R2 != R1) copy_dft<R2>(sm + G::oF2, PR::kFmt == 1 ? 0 : 1);
	for (int e = tid; e < N; e += kThr) {
		const int k1 = e / R2, n2 = e % R2;
		wt[k1 * TWS + n2] = __ldg(tw + (n2 * k1) % N);
	}
	const uint32_t mbar = smem_u32(&mbar_s);
	if (tid == 0) mbar_init(mbar, 1);
	if (tid < 32) tmem_alloc<G::TCOLS>(smem_u32(&tbase_s));
	fence_before_sync();
	__syncthreads();
	fence_after_sync();
	const uint32_t tmem = tbase_s;
	uint32_t phase = 0;
	bool ok = true;
	float2 v[G::NV];
	float inv = 1.f, s = 1.f;
	// tile t -> wave b and first row (row pass) / column (column pass)
	auto decode = [&](long long t, int& b, int& first) {
		b = (int)(t / tt.per_wave);
		const int ti = (int)(t - (long long)b * tt.per_wave);
		first = (COL ? ti : (ti < tt.split ? ti : ti + tt.skip)) * L;
	};
	// input of tile t into v: row pass, set P (x[R2 n1 + n2] of the rows, n1 in
	// the thread's quarter); column pass, set Q (conj of X[k1 + R1 k2] of the
	// columns, k2 in the quarter).  Rows outside the band of live Fourier rows
	// read as zero.
	auto load_tile = [&](long long t) {
		int b, first;
		decode(t, b, first);
		const float2* W = p.work + (long long)b * p.wstride;
		if (!COL) {
			#pragma unroll
			for (int j = 0; j < G::JP; j++) {
				int l, n2;
				G::pinv(lane + kLanes * j, l, n2);
				const int y = first + l;
				const bool live = y <= p.row_k1 || y >= p.row_k2;
				const float2* src = W + (long long)y * N + n2 + R2 * (q * VP);
				#pragma unroll
				for (int i = 0; i < VP; i++) v[j * VP + i] = live ? src[R2 * i] : make_float2(0.f, 0.f);
			}
		}
		else {
			const int nx = p.nx;
			#pragma unroll
			for (int j = 0; j < G::JQ; j++) {
				int l, k1;
				G::qinv(lane + kLanes * j, l, k1);
				const int k20 = q * VQ;
				const float2* src = W + first + (k1 + R1 * k20) * nx + l;
				#pragma unroll
				for (int i = 0; i < VQ; i++) {
					const int y = k1 + R1 * (k20 + i);
					v[j * VQ + i] = (y <= p.in_k1 || y >= p.in_k2) ? conjf2(src[R1 * i * nx]) : make_float2(0.f, 0.f);
				}
			}
		}
	};
	if (blockIdx.x < tt.ntiles) load_tile(blockIdx.x);

	for (long long tile = blockIdx.x; tile < tt.ntiles; tile += gridDim.x) {
		int b, first;
		decode(tile, b, first);
		const long long next = tile + gridDim.x;
		float2* W = p.work + (long long)b * p.wstride;
		if (!COL) {
			// ---- row pass: FT_x -> x P -> IFT_x over rows first .. first + L - 1
			const int row0 = first;
			s = tile_scale<PR>(v, red_s, &inv);
			write_own<R1, G::JP, G::LP, G::SP, PR>(v, ahi, alo, s);
			if (!(ok = stage<R1, G::JP, G::LP, G::SP, PR, DC>(v, ahi, alo, f1, tmem, mbar, phase, inv))) break;
			#pragma unroll
			for (int j = 0; j < G::JP; j++) {
				int l, n2;
				G::pinv(lane + kLanes * j, l, n2);
				#pragma unroll
				for (int i = 0; i < VP; i++) v[j * VP + i] = cmul(v[j * VP + i], wt[(q * VP + i) * TWS + n2]);
			}
			s = tile_scale<PR>(v, red_s, &inv);
			write_pq<G, PR>(v, ahi, alo, s);
			if (!(ok = stage<R2, G::JQ, G::LQ, G::SQ, PR, DC>(v, ahi, alo, f2, tmem, mbar, phase, inv))) break;
			// Fourier space: x P, then the inverse transform through conj(F(conj(.)))
			#pragma unroll
			for (int j = 0; j < G::JQ; j++) {
				int l, k1;
				G::qinv(lane + kLanes * j, l, k1);
				const float2* P = p.mul + (long long)(row0 + l) * N + k1 + R1 * (q * VQ);
				#pragma unroll
				for (int i = 0; i < VQ; i++) v[j * VQ + i] = conjf2(cmul(v[j * VQ + i], __ldg(P + R1 * i)));
			}
			s = tile_scale<PR>(v, red_s, &inv);
			write_own<R2, G::JQ, G::LQ, G::SQ, PR>(v, ahi, alo, s);
			if (!(ok = stage<R2, G::JQ, G::LQ, G::SQ, PR, DC>(v, ahi, alo, f2, tmem, mbar, phase, inv))) break;
			#pragma unroll
			for (int j = 0; j < G::JQ; j++) {
				int l, k1;
				G::qinv(lane + kLanes * j, l, k1);
				#pragma unroll
				for (int i = 0; i < VQ; i++) v[j * VQ + i] = cmul(v[j * VQ + i], wt[k1 * TWS + q * VQ + i]);
			}
			s = tile_scale<PR>(v, red_s, &inv);
			write_qp<G, PR>(v, ahi, alo, s);
			stage_issue<R1, G::JP, G::LP, G::SP, PR, DC>(ahi, alo, f1, tmem, mbar);
			// v is free until the next tile: its loads overlap this last stage
			if (next < tt.ntiles) load_tile(next);
			if (!(ok = stage_wait(mbar, phase))) break;
			#pragma unroll
			for (int j = 0; j < G::JP; j++) {
				int l, n2;
				G::pinv(lane + kLanes * j, l, n2);
				const int y = row0 + l;
				const bool live = y <= p.row_k1 || y >= p.row_k2;
				float2 d[VP];
				tmem_ld_vals<VP, DC>(d_addr<R1>(tmem, j), d, inv);
				if (live) {
					float2* dst = W + (long long)y * N + n2 + R2 * (q * VP);
					#pragma unroll
					for (int i = 0; i < VP; i++) dst[R2 * i] = conjf2(d[i]);
				}
			}
		}
		else {
			// ---- column pass: IFT_y -> x t -> FT_y over columns first .. first + L - 1
			const int nx = p.nx;
			const int col0 = first;
			s = tile_scale<PR>(v, red_s, &inv);
			write_own<R2, G::JQ, G::LQ, G::SQ, PR>(v, ahi, alo, s);
			if (!(ok = stage<R2, G::JQ, G::LQ, G::SQ, PR, DC>(v, ahi, alo, f2, tmem, mbar, phase, inv))) break;
			#pragma unroll
			for (int j = 0; j < G::JQ; j++) {
				int l, k1;
				G::qinv(lane + kLanes * j, l, k1);
				#pragma unroll
				for (int i = 0; i < VQ; i++) v[j * VQ + i] = cmul(v[j * VQ + i], wt[k1 * TWS + q * VQ + i]);
			}
			s = tile_scale<PR>(v, red_s, &inv);
			write_qp<G, PR>(v, ahi, alo, s);
			if (!(ok = stage<R1, G::JP, G::LP, G::SP, PR, DC>(v, ahi, alo, f1, tmem, mbar, phase, inv))) break;
			// real space: x t, then the forward transform
			#pragma unroll
			for (int j = 0; j < G::JP; j++) {
				int l, n2;
				G::pinv(lane + kLanes * j, l, n2);
				const float2* t = p.mul + (p.mul_w ? __ldg(p.mul_w + b) : 0) + col0 + l + (n2 + R2 * (q * VP)) * nx;
				#pragma unroll
				for (int i = 0; i < VP; i++) v[j * VP + i] = cmul(conjf2(v[j * VP + i]), __ldg(t + R2 * i * nx));
			}
			s = tile_scale<PR>(v, red_s, &inv);
			write_own<R1, G::JP, G::LP, G::SP, PR>(v, ahi, alo, s);
			if (!(ok = stage<R1, G::JP, G::LP, G::SP, PR, DC>(v, ahi, alo, f1, tmem, mbar, phase, inv))) break;
			#pragma unroll
			for (int j = 0; j < G::JP; j++) {
				int l, n2;
				G::pinv(lane + kLanes * j, l, n2);
				#pragma unroll
				for (int i = 0; i < VP; i++) v[j * VP + i] = cmul(v[j * VP + i], wt[(q * VP + i) * TWS + n2]);
			}
			s = tile_scale<PR>(v, red_s, &inv);
			write_pq<G, PR>(v, ahi, alo, s);
			stage_issue<R2, G::JQ, G::LQ, G::SQ, PR, DC>(ahi, alo, f2, tmem, mbar);
			// v is free until the next tile: its loads overlap this last stage
			if (next < tt.ntiles) load_tile(next);
			if (!(ok = stage_wait(mbar, phase))) break;
			#pragma unroll
			for (int j = 0; j < G::JQ; j++) {
				int l, k1;
				G::qinv(lane + kLanes * j, l, k1);
				float2 d[VQ];
				tmem_ld_vals<VQ, DC>(d_addr<R2>(tmem, j), d, inv);
				const int k20 = q * VQ;
				float2* dst = W + col0 + (k1 + R1 * k20) * nx + l;
				#pragma unroll
				for (int i = 0; i < VQ; i++) {
					const int y = k1 + R1 * (k20 + i);
					if (y <= p.out_k1 || y >= p.out_k2) dst[R1 * i * nx] = d[i];
				}
			}
		}
	}
	fence_before_sync();
	__syncthreads();
	if (tid < 32) tmem_dealloc<G::TCOLS>(tmem);
	if (!ok && tid == 0 && tt.err) atomicExch(tt.err, 1);
}

template <int N, bool COL, class PR>
cudaError_t launch(const PassArgs& p, TcTiles tt, cudaStream_t s)
{
	using G = Geo<N, COL>;
	auto kern = k_tc_pass<N, COL, PR>;
	static_assert(G::kSmem + 64 <= 227 * 1024, "shared memory");
	// grid size per device, worked out on the first launch on that device
	static int grid_of_dev[64] = {0};
	int dev = 0;
	cudaGetDevice(&dev);
	int& grid = grid_of_dev[dev & 63];
	if (grid == 0) {
		cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, G::kSmem);
		if (e != cudaSuccess) return e;
		int nsm = 0, per_sm = 1;
		cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
		e = resident_ctas(kern, kThr, G::kSmem, 512 / G::TCOLS, &per_sm); // TMEM: 512 columns per SM
		if (e != cudaSuccess) return e;
		grid = nsm * per_sm;
	}
	if (tt.ntiles <= 0) return cudaSuccess;
	kern<<<(unsigned)(tt.ntiles < grid ? tt.ntiles : grid), kThr, G::kSmem, s>>>(p, tt);
	return cudaGetLastError();
}

template <bool COL>
cudaError_t dispatch(int n, const PassArgs& p, const TcTiles& tt, int prec, cudaStream_t s)
{
	const bool f16 = (prec == 2);
	switch (n) {
	case 256: return f16 ? launch<256, COL, Fp16>(p, tt, s) : launch<256, COL, Bf16>(p, tt, s);
	case 512: return f16 ? launch<512, COL, Fp16>(p, tt, s) : launch<512, COL, Bf16>(p, tt, s);
	case 1024: return f16 ? launch<1024, COL, Fp16>(p, tt, s) : launch<1024, COL, Bf16>(p, tt, s);
	case 2048: return f16 ? launch<2048, COL, Fp16>(p, tt, s) : launch<2048, COL, Bf16>(p, tt, s);
	default: return cudaErrorInvalidValue;
	}
}

} // namespace tc

bool tc_supported(int n) { return n == 256 || n == 512 || n == 1024 || n == 2048; }

cudaError_t tc_prepare(cudaStream_t s)
{
	tc::k_build_dft<<<6, tc::kThr, 0, s>>>();
	cudaError_t e = cudaGetLastError();
	if (e != cudaSuccess) return e;
	return cudaStreamSynchronize(s);
}

cudaError_t launch_tc_row(const PassArgs& p, int prec, int* err, cudaStream_t s)
{
	if (!tc_supported(p.nx) || prec < 1 || prec > 2) return cudaErrorInvalidValue;
	const int L = tc::tile_of(p.nx) / p.nx;
	if (p.ny % L) return cudaErrorInvalidValue;
	const int nrb = p.ny / L;
	int split = nrb, skip = 0;
	if (p.row_k1 < p.ny - 1 && p.row_k2 > p.row_k1 + 1) { // row blocks wholly inside the band gap are skipped
		split = p.row_k1 / L + 1;
		const int first_hi = p.row_k2 / L;
		skip = first_hi > split ? first_hi - split : 0;
	}
	tc::TcTiles tt;
	tt.per_wave = nrb - skip;
	tt.ntiles = (long long)tt.per_wave * p.nwave;
	tt.split = split;
	tt.skip = skip;
	tt.err = err;
	return tc::dispatch<false>(p.nx, p, tt, prec, s);
}

cudaError_t launch_tc_col(const PassArgs& p, int prec, int* err, cudaStream_t s)
{
	if (!tc_supported(p.ny) || prec < 1 || prec > 2) return cudaErrorInvalidValue;
	if (p.npgx != p.nx || p.npgy != p.ny) return cudaErrorInvalidValue;
	const int L = tc::tile_of(p.ny) / p.ny;
	if (p.nx % L) return cudaErrorInvalidValue;
	tc::TcTiles tt;
	tt.per_wave = p.nx / L;
	tt.ntiles = (long long)tt.per_wave * p.nwave;
	tt.err = err;
	return tc::dispatch<true>(p.ny, p, tt, prec, s);
}

} // namespace jms
