// jms_passes.cuh -- fused FP32 multislice pass kernels (templates) for sm_100a.
//
// Included by the jms_inst_*.cu files, which instantiate the launchers for
// their share of the supported line lengths; jms_kernels.cu dispatches on the
// grid size.  See jms_kernels.h for the pass structure and jms_fft.cuh for the
// in-register DFTs.  Reference semantics followed here:
//   slice loop order          src/JMultiSlice.cpp:4590-4651 (GPUMultislice)
//   Fourier-space readout     src/JMultiSlice.cpp:4218-4367 (ReadoutDifDet_d)
//   real-space readout        src/JMultiSlice.cpp:4369-4465 (ReadoutImgDet_d)
//   grating multiply          src/cu/ArrayOps.cu:202-234 (MulKernel / sub-frame)
//   probe offset              src/JMultiSlice.cpp:1961-2084, src/cu/ArrayOps.cu:340-421
//
// Line transforms.  A line of N = A*B points is held by B threads, thread j
// owning x[j + B m] (m < A): loads and stores of that layout are coalesced.
// A transform runs in two register stages around one shared-memory exchange
// and leaves the line in a "middle" layout, where the pass applies its
// elementwise work (x P and Fourier readout, or real-space readout and x t);
// the opposite-direction transform then returns the line to the load layout.
//   split 1 (A, B any):  the middle layout has A threads per line, thread k1
//       holding X[k1 + A k2] (k2 < B); threads k1 >= A idle in the middle.
//   split 2 (B = 2A):   the B-point stage is shared by a thread pair with a
//       radix-2 step over warp shuffles, so every thread keeps A values in all
//       stages: thread (k1, h) = 2 k1 + h holds X[k1 + A (k + A h)], k < A.
// In the row passes a line whose threads fit in one warp in every stage
// (split 2, split 1 with A = B, and split 1 with B > A on a row tile of B
// threads per line) exchanges under warp barriers only, so the warps of a CTA
// run their lines independently; column lines span the CTA's warps and take
// CTA barriers.  Stage twiddles come from a shared copy (TwShared) where the
// plan's table layout allows it.
#pragma once
#include "jms_fft.cuh"
#include "jms_kernels.h"
#include "jms_sizes.h"

namespace jms {

// ---------------------------------------------------------------------------
// tiles: thread <-> (line, position) maps and exchange-buffer layouts
// ---------------------------------------------------------------------------
// Row tile: LINES rows per CTA; thread t -> (line t / P, position t % P) for a
// role of P threads per line, or (line t / W, position t % W) in every role
// when the tile has a fixed line width W (positions P ... W - 1 then idle).
template <int LINES, int W = 0>
struct RowTile {
	static constexpr int kLines = LINES;
	static constexpr int kWidth = W;
	static constexpr int kPartner = 1;   // lane distance of positions 2k and 2k+1
	template <int P>
	__device__ __forceinline__ static void role(int tid, int& line, int& pos)
	{
		static_assert(W == 0 || P <= W, "a role wider than the tile's lines");
		constexpr int Q = W > 0 ? W : P;
		line = tid / Q;
		pos = tid % Q;
	}
	// Lines of P threads (P dividing 32) lie inside one warp, and so do their
	// exchange regions: a transform whose stages keep that role needs only
	// warp barriers, and the warps of a CTA run their lines independently.
	template <int P>
	__host__ __device__ static constexpr bool warp_lines() { return 32 % (W > 0 ? W : P) == 0; }
	// split 1 exchange S(line, k1, j), k1 < A, j < B, rows padded to B+1.  A
	// line's region has the same size for <A, B> and <B, A> (the forward and
	// inverse exchanges), so with warp-local lines one line's inverse exchange
	// never writes into another line's forward exchange.
	template <int A, int B>
	__host__ __device__ static constexpr int pad_line() { return A * (B + 1) > B * (A + 1) ? A * (B + 1) : B * (A + 1); }
	template <int A, int B>
	__device__ __forceinline__ static int s_pad(int line, int k1, int j) { return line * pad_line<A, B>() + k1 * (B + 1) + j; }
	template <int A, int B>
	static constexpr int sm_pad() { return LINES * pad_line<A, B>(); }
	// split 2 exchanges S(line, a, b), a < A, b < B, rows padded to B+2: the
	// pair reads of a half warp (a = 0..7, b = 2i + h) land on 16 distinct
	// bank pairs, and every per-thread loop has a constant address stride
	//   forward: a = k1, b = j (written by j, read by the pair (k1, h) at j = 2i + h)
	//   inverse: a = n1, b = q2 (written by the pair (n1, h) at q2 = 2m + h, read by q2)
	template <int A, int B>
	__device__ __forceinline__ static int s_fwd(int line, int a, int b) { return (line * A + a) * (B + 2) + b; }
	template <int A, int B>
	__device__ __forceinline__ static int s_inv(int line, int q2, int n1) { return (line * A + n1) * (B + 2) + q2; }
	template <int A, int B>
	static constexpr int sm_split() { return LINES * A * (B + 2); }
	// 3-stage exchanges for N = R^3 (see fft3): S1(line, k1, t) and
	// S2(line, k1, k2, j) in separate regions; the strides make the 16 lanes
	// of a half warp (k1 = t mod R fastest) hit distinct bank pairs
	template <int R>
	__host__ __device__ static constexpr int s3a_row() { return R * R + ((16 / R - R * R) % 16 + 16) % 16; }   // = 16/R mod 16
	template <int R>
	__host__ __device__ static constexpr int s3b_j() { return R + ((1 - R) % 16 + 16) % 16; }                    // = 1 mod 16
	template <int R>
	__host__ __device__ static constexpr int s3b_k1()
	{
		constexpr int base = R * s3b_j<R>();
		return base + ((16 / R - base) % 16 + 16) % 16;                                          // = 16/R mod 16
	}
	template <int R>
	__host__ __device__ static constexpr int s3_line() { return R * s3a_row<R>() + R * s3b_k1<R>(); }
	template <int R>
	__device__ __forceinline__ static int s3a(int line, int k1, int t) { return line * s3_line<R>() + k1 * s3a_row<R>() + t; }
	template <int R>
	__device__ __forceinline__ static int s3b(int line, int k1, int k2, int j)
	{
		return line * s3_line<R>() + R * s3a_row<R>() + k1 * s3b_k1<R>() + k2 * s3b_j<R>() + j;
	}
	template <int R>
	static constexpr int sm3() { return LINES * s3_line<R>(); }
};

// Column tile: C columns per CTA; thread t -> (column t % C, position t / C),
// so a warp touches C consecutive complex values of a few rows.  Exchange
// buffers keep the column index fastest; a pad of C complex per k1 block keeps
// the k1 groups of a half warp on distinct banks when C < 16.
template <int C>
struct ColTile {
	static constexpr int kLines = C;
	static constexpr int kPartner = C;
	static constexpr int PAD = (C < 16) ? C : 0;
	static constexpr int kWidth = 0;
	template <int P>
	__device__ __forceinline__ static void role(int tid, int& line, int& pos) { line = tid % C; pos = tid / C; }
	template <int P>
	__host__ __device__ static constexpr bool warp_lines() { return false; }   // a column's positions span warps
	template <int A, int B>
	__device__ __forceinline__ static int s_pad(int line, int k1, int j) { return k1 * (B * C + PAD) + j * C + line; }
	template <int A, int B>
	static constexpr int sm_pad() { return A * (B * C + PAD); }
	template <int A, int B>
	__device__ __forceinline__ static int s_fwd(int line, int k1, int j) { return k1 * (B * C + PAD) + j * C + line; }
	template <int A, int B>
	__device__ __forceinline__ static int s_inv(int line, int q2, int n1) { return n1 * (B * C + PAD) + q2 * C + line; }
	template <int A, int B>
	static constexpr int sm_split() { return A * (B * C + PAD); }
	// 3-stage exchanges: S1(c, k1, t) then S2(c, k1, k2, j), column fastest
	template <int R>
	__device__ __forceinline__ static int s3a(int line, int k1, int t) { return k1 * (R * R * C + PAD) + t * C + line; }
	template <int R>
	__device__ __forceinline__ static int s3b(int line, int k1, int k2, int j)
	{
		return R * (R * R * C + PAD) + k1 * (R * R * C + PAD) + (k2 * R + j) * C + line;
	}
	template <int R>
	static constexpr int sm3() { return 2 * R * (R * R * C + PAD); }
};

// Barrier around an exchange of lines of P threads: a warp barrier (which also
// orders the warp's shared-memory accesses) when every line and its exchange
// region lie inside one warp, else a CTA barrier.
template <class Tile, int P>
__device__ __forceinline__ void line_sync()
{
	if constexpr (Tile::template warp_lines<P>()) __syncwarp();
	else __syncthreads();
}

// twiddle by table value w = exp(-2 pi i k / N) (conjugated for the inverse)
template <bool INV>
__device__ __forceinline__ float2 tw_mul(float2 v, float2 w) { return INV ? cmulc(v, w) : cmul(v, w); }

// Stage twiddles W_N^(a b), a on the A-point side of a plan and b on the
// B-point side: from the N-entry table in global memory (read-only path), or
// from a CTA's shared copy laid out [a][b] with rows padded to B+2.  A 64-bit
// shared access is served per half warp, whose 16 lanes need distinct bank
// pairs: reading W^(k1 j) over consecutive j they have them for any row
// length, and reading W^(n1 q2) over the pairs (n1 < 8, h; q2 = 2m + h) they
// sit at (B+2) n1 + h + 2m, distinct modulo 16 because B + 2 = 2 mod 16 for
// B = 8, 16, 32, 64 (with rows of B+1 the lanes (n1, 1) and (n1 + 1, 0)
// collided, doubling the wavefronts).
struct TwGlobal {
	const float2* p;
	__device__ __forceinline__ float2 operator()(int a, int b) const { return __ldg(p + a * b); }
};
template <int B>
struct TwShared {
	const float2* s;
	__device__ __forceinline__ float2 operator()(int a, int b) const { return s[a * (B + 2) + b]; }
};
// Fills a shared [A][B+2] twiddle copy from the global table; the caller
// places a CTA barrier before its first use.
template <int A, int B, int NT>
__device__ __forceinline__ void fill_tw_shared(float2* tws, const float2* __restrict__ tw, int tid)
{
	for (int i = tid; i < A * (B + 2); i += NT) {
		const int a = i / (B + 2), b = i - a * (B + 2);
		tws[i] = b < B ? __ldg(tw + a * b) : make_float2(0.f, 0.f);
	}
}

// ---- split 1 -----------------------------------------------------------------
// in: B threads/line, thread j holds x[j + B m] (m < A)
// out: A threads/line, thread k1 holds X[k1 + A k2] (k2 < B)
template <int A, int B, bool INV, class Tile, int RM, class TW>
__device__ __forceinline__ void fft_s1_fwd(float2 (&v)[RM], float2* sm, const TW& tw, int tid)
{
	int line, j;
	Tile::template role<B>(tid, line, j);
	const bool in_role = line < Tile::kLines && j < B;
	if (in_role) {
		dft_reg<A, 1, 0, INV>(v);
		#pragma unroll
		for (int k1 = 1; k1 < A; k1++) v[k1] = tw_mul<INV>(v[k1], tw(k1, j));
		#pragma unroll
		for (int k1 = 0; k1 < A; k1++) sm[Tile::template s_pad<A, B>(line, k1, j)] = v[k1];
	}
	// with A = B, or a tile whose lines keep max(A, B) threads in every role,
	// both stages give a line the same threads, so a line inside a warp
	// exchanges under a warp barrier
	constexpr int P = A > B ? A : B;
	constexpr bool same = A == B || Tile::kWidth >= P;
	if constexpr (same) line_sync<Tile, P>();
	else __syncthreads();
	Tile::template role<A>(tid, line, j);
	if (line < Tile::kLines && j < A) {
		#pragma unroll
		for (int jj = 0; jj < B; jj++) v[jj] = sm[Tile::template s_pad<A, B>(line, j, jj)];
		dft_reg<B, 1, 0, INV>(v);
	}
	if constexpr (same) line_sync<Tile, P>();
	else __syncthreads();
}

// in: A threads/line, thread k1 holds x[k1 + A k2] (k2 < B)
// out: B threads/line, thread j holds y[j + B m] (m < A)
template <int A, int B, bool INV, class Tile, int RM, class TW>
__device__ __forceinline__ void fft_s1_inv(float2 (&v)[RM], float2* sm, const TW& tw, int tid)
{
	// the transpose of fft_s1_fwd: per-thread B-point DFT, exchange, A-point DFT
	fft_s1_fwd<B, A, INV, Tile>(v, sm, tw, tid);
}

// ---- split 2 (B = 2A) ------------------------------------------------------------
// in: B threads/line, thread j holds x[j + B m] (m < A)
// out: B threads/line, thread (k1, h) = 2 k1 + h holds X[k1 + A (k + A h)] (k < A)
template <int A, bool INV, class Tile, int RM, class TW>
__device__ __forceinline__ void fft_s2_fwd(float2 (&v)[RM], float2* sm, const TW& tw, int tid)
{
	constexpr int B = 2 * A;
	int line, j;
	Tile::template role<B>(tid, line, j);
	dft_reg<A, 1, 0, INV>(v);
	#pragma unroll
	for (int k1 = 1; k1 < A; k1++) v[k1] = tw_mul<INV>(v[k1], tw(k1, j));
	#pragma unroll
	for (int k1 = 0; k1 < A; k1++) sm[Tile::template s_fwd<A, B>(line, k1, j)] = v[k1];
	line_sync<Tile, B>();
	const int k1 = j >> 1, h = j & 1;
	#pragma unroll
	for (int i = 0; i < A; i++) v[i] = sm[Tile::template s_fwd<A, B>(line, k1, 2 * i + h)];
	dft_reg<A, 1, 0, INV>(v);
	// radix-2 across the pair: Y[k] = E[k] + W_B^k O[k], Y[k + A] = E[k] - W_B^k O[k].
	// The odd thread twiddles its own value before the exchange, so both
	// threads finish with one sign-weighted add: u + o (h = 0), o - u (h = 1).
	const float sgn = h ? -1.f : 1.f;
	static_for<A>([&](auto K) {
		constexpr int k = K.value;
		const float2 u = h ? twiddle_ct<k, B, INV>(v[k]) : v[k];
		float2 o;
		o.x = __shfl_xor_sync(0xffffffffu, u.x, Tile::kPartner);
		o.y = __shfl_xor_sync(0xffffffffu, u.y, Tile::kPartner);
		v[k] = __ffma2_rn(make_float2(sgn, sgn), u, o);
	});
	line_sync<Tile, B>();
}

// in: B threads/line, thread (n1, h) = 2 n1 + h holds x[n1 + A (k + A h)] (k < A)
// out: B threads/line, thread j holds y[j + B m] (m < A)
template <int A, bool INV, class Tile, int RM, class TW>
__device__ __forceinline__ void fft_s2_inv(float2 (&v)[RM], float2* sm, const TW& tw, int tid)
{
	constexpr int B = 2 * A;
	int line, j;
	Tile::template role<B>(tid, line, j);
	const int n1 = j >> 1, h = j & 1;
	// radix-2 decimation in frequency over n2 = k + A h across the pair:
	// v + o (h = 0), W_B^k (o - v) (h = 1)
	const float sgn = h ? -1.f : 1.f;
	static_for<A>([&](auto K) {
		constexpr int k = K.value;
		float2 o;
		o.x = __shfl_xor_sync(0xffffffffu, v[k].x, Tile::kPartner);
		o.y = __shfl_xor_sync(0xffffffffu, v[k].y, Tile::kPartner);
		const float2 d = __ffma2_rn(make_float2(sgn, sgn), v[k], o);
		v[k] = h ? twiddle_ct<k, B, INV>(d) : d;
	});
	dft_reg<A, 1, 0, INV>(v);   // output q2 = 2 m + h
	#pragma unroll
	for (int m = 0; m < A; m++) {
		const int q2 = 2 * m + h;
		if (n1 > 0) v[m] = tw_mul<INV>(v[m], tw(n1, q2));
		sm[Tile::template s_inv<A, B>(line, q2, n1)] = v[m];
	}
	line_sync<Tile, B>();
	#pragma unroll
	for (int i = 0; i < A; i++) v[i] = sm[Tile::template s_inv<A, B>(line, j, i)];
	dft_reg<A, 1, 0, INV>(v);
	line_sync<Tile, B>();
}

// ---- 3 stages, N = R^3 ---------------------------------------------------------
// T = R^2 threads per line; thread t holds x[t + T m] (m < R) on entry and
// X[t + T k3] (k3 < R) on exit, so the transform maps its layout onto itself.
//   stage A: R-point DFT over m, twiddle W_N^(t k1), exchange S1;
//   stage B: thread (k1 = t mod R, j = t / R) takes Y[k1][j + R m'], R-point
//            DFT over m', twiddle W_N^(R j k2), exchange S2;
//   stage C: thread (k1, k2 = t / R) takes the R values over j, R-point DFT.
// S1 and S2 are separate regions, so two barriers per transform suffice.
template <int R, bool INV, class Tile, int RM, class TW>
__device__ __forceinline__ void fft3(float2 (&v)[RM], float2* sm, const TW& tw, int tid)
{
	constexpr int T = R * R;
	int line, t;
	Tile::template role<T>(tid, line, t);
	dft_reg<R, 1, 0, INV>(v);
	#pragma unroll
	for (int k1 = 1; k1 < R; k1++) v[k1] = tw_mul<INV>(v[k1], tw(t, k1));
	#pragma unroll
	for (int k1 = 0; k1 < R; k1++) sm[Tile::template s3a<R>(line, k1, t)] = v[k1];
	line_sync<Tile, T>();
	const int k1 = t % R, jj = t / R;
	#pragma unroll
	for (int m = 0; m < R; m++) v[m] = sm[Tile::template s3a<R>(line, k1, jj + R * m)];
	dft_reg<R, 1, 0, INV>(v);
	#pragma unroll
	for (int k2 = 1; k2 < R; k2++) v[k2] = tw_mul<INV>(v[k2], tw(R * jj, k2));
	#pragma unroll
	for (int k2 = 0; k2 < R; k2++) sm[Tile::template s3b<R>(line, k1, k2, jj)] = v[k2];
	line_sync<Tile, T>();
	#pragma unroll
	for (int j = 0; j < R; j++) v[j] = sm[Tile::template s3b<R>(line, k1, jj, j)];
	dft_reg<R, 1, 0, INV>(v);
}

// ---- plans -------------------------------------------------------------------------
template <int A_, int B_, int CC_>
struct Plan {
	static constexpr int A = A_, B = B_, N = A_ * B_;
	static constexpr int S = (B_ == 2 * A_ && A_ >= 4) ? 2 : 1;
	static constexpr int RM = (S == 2) ? A_ : (A_ > B_ ? A_ : B_);   // registers per thread (complex)
	static constexpr int T = B_;                                       // threads per line (load layout)
	static constexpr int TMID = (S == 2) ? B_ : A_;                    // threads per line (middle layout)
	static constexpr int EMID = (S == 2) ? A_ : B_;                    // values per thread (middle layout)
	static constexpr int TMAX = (T > TMID) ? T : TMID;
	static constexpr int CC = CC_;                                     // columns per column-pass CTA
	// the passes keep a shared [A][B+2] copy of the stage twiddles (split 2,
	// and split 1 with A = B, whose inverse indexes the table the same way)
	static constexpr bool SMEM_TW = (S == 2 || A_ == B_);
	static constexpr int TWS = SMEM_TW ? A_ * (B_ + 2) : 1;
	// line index of the e-th middle value of position pos
	__device__ __forceinline__ static int mid(int pos, int e)
	{
		if constexpr (S == 2) return (pos >> 1) + A * (e + A * (pos & 1));
		else return pos + A * e;
	}
	template <bool INV, class Tile, class TW>
	__device__ __forceinline__ static void to_mid(float2 (&v)[RM], float2* sm, const TW& tw, int tid)
	{
		if constexpr (S == 2) fft_s2_fwd<A, INV, Tile>(v, sm, tw, tid);
		else fft_s1_fwd<A, B, INV, Tile>(v, sm, tw, tid);
	}
	template <bool INV, class Tile, class TW>
	__device__ __forceinline__ static void from_mid(float2 (&v)[RM], float2* sm, const TW& tw, int tid)
	{
		if constexpr (S == 2) fft_s2_inv<A, INV, Tile>(v, sm, tw, tid);
		else fft_s1_inv<A, B, INV, Tile>(v, sm, tw, tid);
	}
	// Threads per line of the row tile in every role: a split-1 plan with
	// B > A gives its middle role (A threads) the load role's B threads, A of
	// them active, so a line keeps its threads through both stages; 0 (the
	// role's own count) otherwise.  A CTA holds as many threads either way.
	static constexpr int ROWW = (S == 1 && B_ > A_) ? B_ : 0;
	// every exchange of to_mid / from_mid takes only warp barriers (a split-1
	// plan with A > B changes the threads of a line between its stages and
	// keeps CTA barriers)
	template <class Tile>
	__host__ __device__ static constexpr bool warp_local()
	{
		if constexpr (S == 2 || A_ == B_) return Tile::template warp_lines<B>();
		else return Tile::kWidth == B_ && B_ > A_ && Tile::template warp_lines<B>();
	}
	template <class Tile>
	static constexpr int smem_elems()
	{
		if constexpr (S == 2) return Tile::template sm_split<A, B>();
		else {
			constexpr int a = Tile::template sm_pad<A, B>(), b = Tile::template sm_pad<B, A>();
			return a > b ? a : b;
		}
	}
};

// Three equal radices: N = R^3, R^2 threads per line with R values each; the
// middle layout equals the load layout.
template <int R_, int CC_ = 8>
struct Plan3 {
	static constexpr int R = R_, N = R_ * R_ * R_;
	static constexpr int A = R_, B = R_ * R_;            // load layout: thread j holds x[j + B m], m < A
	static constexpr int RM = R_, T = B, TMID = B, EMID = R_, TMAX = B;
	static constexpr int CC = CC_;
	static constexpr int ROWW = 0;
	static constexpr bool SMEM_TW = false;
	static constexpr int TWS = 1;
	__device__ __forceinline__ static int mid(int pos, int e) { return pos + B * e; }
	template <bool INV, class Tile, class TW>
	__device__ __forceinline__ static void to_mid(float2 (&v)[RM], float2* sm, const TW& tw, int tid)
	{
		fft3<R_, INV, Tile>(v, sm, tw, tid);
	}
	template <bool INV, class Tile, class TW>
	__device__ __forceinline__ static void from_mid(float2 (&v)[RM], float2* sm, const TW& tw, int tid)
	{
		// the second transform writes S1 before its first barrier; the barriers
		// of the first transform already ordered all reads of S1 before it
		fft3<R_, INV, Tile>(v, sm, tw, tid);
	}
	template <class Tile>
	__host__ __device__ static constexpr bool warp_local() { return Tile::template warp_lines<B>(); }
	template <class Tile>
	static constexpr int smem_elems() { return Tile::template sm3<R_>(); }
};

__host__ __device__ constexpr int gcd_ct(int a, int b) { return b == 0 ? a : gcd_ct(b, a % b); }
// rows per row-pass CTA: about 256 threads, a whole number of warps
template <class PL>
__host__ __device__ constexpr int row_lines()
{
	constexpr int T = PL::TMAX;
	constexpr int m = 32 / gcd_ct(T, 32);
	constexpr int l = (256 / T) / m * m;
	return l < m ? m : l;
}
// the row tile of a plan
template <class PL>
using RowTileOf = RowTile<row_lines<PL>(), PL::ROWW>;

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

// Scrambled pixel index at which psi(ky = y, kx) is read out, after the
// integer-pixel diffraction descan (DescanDifN, src/JMultiSlice.cpp:2184-2273:
// psi(kx, ky) is read out at pixel (kx - dnx, ky - dny), periodic)
__device__ __forceinline__ void readout_pixel(const PassArgs& p, int& y, int& kx)
{
	if (p.descan_x | p.descan_y) {
		kx -= p.descan_x; kx %= p.nx; if (kx < 0) kx += p.nx;
		y -= p.descan_y; y %= p.ny; if (y < 0) y += p.ny;
	}
}

// Fourier-space readout of one element psi(ky = y, kx) of wave b
// (ReadoutDifDet_d, src/JMultiSlice.cpp:4277-4359) except the integrating
// detectors: diffraction and wave channels, binned pattern.
__device__ __forceinline__ void readout_fourier_channels(const PassArgs& p, int b, int y, int kx, float2 v)
{
	const long long N = (long long)p.nx * p.ny;
	readout_pixel(p, y, kx);
	const int idx = y * p.nx + kx;                    // nx * ny < 2^31
	const float pw = cnorm(v);
	const long long c = (long long)b * p.chan_wstride + (long long)p.plane * N + idx;
	if (p.dif) p.dif[c] += p.weight * pw;
	if (p.dif_avg) p.dif_avg[c] += p.weight * pw;
	if (p.wff) p.wff[c] = __ffma2_rn(v, make_float2(p.weight, p.weight), p.wff[c]);
	if (p.wff_avg) p.wff_avg[c] = __ffma2_rn(v, make_float2(p.weight, p.weight), p.wff_avg[c]);
	if (p.bin_out && p.plane == p.bin_plane) {
		// unscrambled position (zero beam at nx/2, ny/2 as GetUnscrambleHash,
		// src/JMultiSlice.cpp:1932-1958), then bin x bin pixel blocks
		int ux = kx + (p.nx >> 1); if (ux >= p.nx) ux -= p.nx;
		int uy = y + (p.ny >> 1); if (uy >= p.ny) uy -= p.ny;
		int bx = ux / p.bin, by = uy / p.bin;
		const int bp = p.wave_pos > 0 ? b % p.wave_pos : b;   // the wave's probe position
		if (bx < p.nbx && by < p.nby)
			atomicAdd(p.bin_out + ((long long)bp * p.nby + by) * p.nbx + bx, p.weight * pw);
	}
}

// Fourier-space readout of one element psi(ky = y, kx) of wave b
// (ReadoutDifDet_d, src/JMultiSlice.cpp:4277-4359): integrating detectors
// into acc, then the channels.
__device__ __forceinline__ void readout_fourier(const PassArgs& p, int b, int y, int kx, float2 v,
	float (&acc)[kMaxDet])
{
	int yd = y, kxd = kx;
	readout_pixel(p, yd, kxd);
	const int idx = yd * p.nx + kxd;                  // nx * ny < 2^31
	const float pw = cnorm(v);
	const float* det = p.det + idx;
	const int N = p.nx * p.ny;
	#pragma unroll
	for (int d = 0; d < kMaxDet; d++)
		if (d < p.ndet) acc[d] = fmaf(pw, __ldg(det + d * N), acc[d]);
	readout_fourier_channels(p, b, y, kx, v);
}

// Real-space readout of psi(y, x) of wave b (ReadoutImgDet_d, src/JMultiSlice.cpp:4392-4459).
__device__ __forceinline__ void readout_real(const PassArgs& p, int b, int y, int x, float2 v)
{
	const long long N = (long long)p.nx * p.ny;
	const long long c = (long long)b * p.chan_wstride + (long long)p.plane * N + (long long)y * p.nx + x;
	const float pw = cnorm(v);
	if (p.img) p.img[c] += p.weight * pw;
	if (p.img_avg) p.img_avg[c] += p.weight * pw;
	if (p.wfr) p.wfr[c] = __ffma2_rn(v, make_float2(p.weight, p.weight), p.wfr[c]);
	if (p.wfr_avg) p.wfr_avg[c] = __ffma2_rn(v, make_float2(p.weight, p.weight), p.wfr_avg[c]);
}

// offset phase plate exp(-i (2 pi turns + cppl)) at scrambled pixel (i, j);
// turns = fi dx/a + fj dy/b + fz (fi^2/a^2 + fj^2/b^2) is formed in FP64 and
// reduced mod 1 before the FP32 sincos (large k.dx phases keep full accuracy).
__device__ __forceinline__ float2 offset_factor(const double* sh, int i, int j, int nx, int ny, float cp)
{
	// signed frequency index (i + n/2) mod n - n/2 of bin i < n, without a division
	const int fi = i < nx - (nx >> 1) ? i : i - nx;
	const int fj = j < ny - (ny >> 1) ? j : j - ny;
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
// pass kernels (template parameter: the line plan of the transformed axis)
// ---------------------------------------------------------------------------
// Entry row pass: [offset] -> Fourier readout (plane) -> IFT_x.
template <class PL>
__global__ void __launch_bounds__(row_lines<PL>() * PL::TMAX)
k_entry_rows(const PassArgs p)
{
	constexpr int N = PL::N, L = row_lines<PL>(), NT = L * PL::TMAX;
	using T = RowTileOf<PL>;
	extern __shared__ float2 sm[];
	const int tid = threadIdx.x, b = blockIdx.y, row0 = blockIdx.x * L;
	const int nval = min(L, p.ny - row0);
	// Rows outside the source's band of live rows (row_k1 / row_k2: the
	// incident wave's all-zero rows, for scans without beam tilt) are zero: a
	// CTA of such rows does nothing, and they are neither read, read out nor
	// stored (the first column pass reads them as zero).
	if (row0 > p.row_k1 && row0 + nval - 1 < p.row_k2) return;
	float2* W = p.work + (long long)b * p.wstride;
	float2 v[PL::RM];
	#pragma unroll
	for (int m = 0; m < PL::RM; m++) v[m] = make_float2(0.f, 0.f);
	float acc[kMaxDet];
	#pragma unroll
	for (int d = 0; d < kMaxDet; d++) acc[d] = 0.f;
	int line, j;
	T::template role<PL::T>(tid, line, j);
	if (line < nval && (row0 + line <= p.row_k1 || row0 + line >= p.row_k2)) {
		const int y = row0 + line;
		#pragma unroll
		for (int m = 0; m < PL::A; m++) {
			const int kx = j + PL::B * m;
			float2 a;
			if (p.shift) {
				int sx = kx, sy = y;
				if (p.ibtx | p.ibty) {   // beam tilt: a periodic shift of the incident wave (uniform branch)
					sx -= p.ibtx; sx %= N; if (sx < 0) sx += N;
					sy -= p.ibty; sy %= p.ny; if (sy < 0) sy += p.ny;
				}
				a = __ldg(p.wav0 + (long long)sy * N + sx);
				// the offset phase only where the probe is nonzero (inside its aperture)
				if (a.x != 0.f || a.y != 0.f) {
					const float cp = p.cppl ? __ldg(p.cppl + (long long)y * N + kx) : 0.f;
					a = cmul(a, offset_factor(p.shift + 4 * b, kx, y, N, p.ny, cp));
				}
			}
			else {
				a = p.wav0 ? __ldg(p.wav0 + (long long)y * N + kx) : W[(long long)y * N + kx];
			}
			if (p.plane >= 0) readout_fourier(p, b, y, kx, a, acc);
			v[m] = a;
		}
	}
	if (p.plane >= 0 && p.ndet > 0) block_store_partials<NT>(acc, p, b);
	PL::template to_mid<true, T>(v, sm, TwGlobal{p.twx}, tid);
	int pos;
	T::template role<PL::TMID>(tid, line, pos);
	if (line < nval && pos < PL::TMID && (row0 + line <= p.row_k1 || row0 + line >= p.row_k2)) {
		float2* dst = W + (long long)(row0 + line) * N;
		#pragma unroll
		for (int e = 0; e < PL::EMID; e++) dst[PL::mid(pos, e)] = v[e];
	}
}

// Row pass: FT_x -> x P -> Fourier readout (plane) -> IFT_x.  READ selects
// the variant with the readout code (used at readout planes only, as the
// kernel k_row_pass_read with launch bounds of its own), so the steps without
// readout do not carry its registers.
template <class PL, bool READ>
__device__ __forceinline__ void row_pass_body(const PassArgs& p)
{
	constexpr int N = PL::N, L = row_lines<PL>(), NT = L * PL::TMAX;
	using T = RowTileOf<PL>;
	extern __shared__ float2 sm[];
	const int tid = threadIdx.x, b = blockIdx.y, row0 = blockIdx.x * L;
	const int nval = min(L, p.ny - row0);
	// rows outside the propagator's band end up exactly zero: a CTA whose rows
	// are all outside does nothing, and such rows are neither read nor stored
	// (the column pass reads them as zero)
	if (row0 > p.row_k1 && row0 + nval - 1 < p.row_k2) return;
	__shared__ float2 tws[PL::TWS];
	const auto tw = [&] {
		if constexpr (PL::SMEM_TW) return TwShared<PL::B>{tws};
		else return TwGlobal{p.twx};
	}();
	float2* W = p.work + (long long)b * p.wstride;
	float2 v[PL::RM];
	#pragma unroll
	for (int m = 0; m < PL::RM; m++) v[m] = make_float2(0.f, 0.f);
	int line, j;
	T::template role<PL::T>(tid, line, j);
	const int yl = row0 + line;
	const bool live = line < nval && (yl <= p.row_k1 || yl >= p.row_k2);
	if (live) {
		const float2* src = W + (long long)yl * N;
		#pragma unroll
		for (int m = 0; m < PL::A; m++) v[m] = src[j + PL::B * m];
	}
	// the twiddle copy is filled while the row loads are in flight, so the
	// barrier waits for both latencies at once
	if constexpr (PL::SMEM_TW) {
		fill_tw_shared<PL::A, PL::B, NT>(tws, p.twx, tid);
		__syncthreads();
	}
	// with warp-local lines and no CTA-wide readout, a warp whose lines are
	// all dead (band gap, past the last row) has nothing more to do
	if constexpr (!READ && PL::template warp_local<T>())
		if (__all_sync(0xffffffffu, !live)) return;
	PL::template to_mid<false, T>(v, sm, tw, tid);
	{
		int pos;
		T::template role<PL::TMID>(tid, line, pos);
		const bool mid_live = line < nval && pos < PL::TMID;
		const int y = row0 + line;
		if (mid_live) {
			const float2* P = p.mul + (long long)y * N;
			#pragma unroll
			for (int e = 0; e < PL::EMID; e++) v[e] = cmul(v[e], __ldg(P + PL::mid(pos, e)));
		}
		if (READ) {
			// channels in a loop of their own (uniform test), so their
			// registers do not add to those of the propagator loads
			const bool chan = p.dif || p.dif_avg || p.wff || p.wff_avg || (p.bin_out && p.plane == p.bin_plane);
			if (chan && mid_live) {
				#pragma unroll
				for (int e = 0; e < PL::EMID; e++) readout_fourier_channels(p, b, y, PL::mid(pos, e), v[e]);
			}
			// integrating detectors one at a time (a rolled loop): unrolled
			// over the detectors, the compiler kept every element's detector
			// loads in flight (128 registers, half the plain pass's occupancy).
			// Each warp's sums wait in shared memory for one CTA barrier after
			// the last detector; the per-warp and per-CTA summation orders are
			// those of block_store_partials.
			__shared__ float red[NT / 32][kMaxDet];
			const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
			for (int d = 0; d < p.ndet; d++) {
				float s = 0.f;
				if (mid_live) {
					const float* det = p.det + (long long)d * p.nx * p.ny;   // detector d: [ny][nx]
					#pragma unroll
					for (int e = 0; e < PL::EMID; e++) {
						int yd = y, kx = PL::mid(pos, e);
						readout_pixel(p, yd, kx);
						s = fmaf(cnorm(v[e]), __ldg(det + yd * p.nx + kx), s);
					}
				}
				s = warp_sum(s);
				if (lane == 0) red[warp][d] = s;
			}
			if (p.ndet > 0) {
				__syncthreads();
				if ((int)threadIdx.x < p.ndet) {
					float t = 0.f;
					#pragma unroll
					for (int w = 0; w < NT / 32; w++) t += red[w][threadIdx.x];
					p.partial[(((long long)b * p.ndetslc + p.plane) * p.ndet + threadIdx.x) * p.nblk + blockIdx.x] = t;
				}
			}
		}
	}
	if (!p.store) return;
	PL::template from_mid<true, T>(v, sm, tw, tid);
	if (live) {
		float2* dst = W + (long long)yl * N;
		#pragma unroll
		for (int m = 0; m < PL::A; m++) dst[j + PL::B * m] = v[m];
	}
}

// Resident CTAs asked of the readout kernel: for plans of at most 16 values
// a thread (whose plain pass takes 64 registers) the plain pass's count, so
// the readout code spills a few bytes instead of halving the occupancy;
// larger plans are held to about 112 registers.
template <class PL>
__host__ __device__ constexpr int read_min_blocks()
{
	return 65536 / (row_lines<PL>() * PL::TMAX * (PL::RM <= 16 ? 64 : 112)) > 0
		? 65536 / (row_lines<PL>() * PL::TMAX * (PL::RM <= 16 ? 64 : 112)) : 1;
}
// Resident CTAs asked of a plain pass of NT threads: the count at 64
// registers for plans of at most 16 values a thread, at 128 for larger ones.
// Left free, the compiler took 70 (512 rows), 142 (1024 rows) and 140 (1024
// columns) once the lines ran warp by warp and the twiddles came from shared
// memory, each dropping a resident CTA.
template <class PL, int NT>
__host__ __device__ constexpr int pass_min_blocks()
{
	return 65536 / (NT * (PL::RM <= 16 ? 64 : 128)) > 0 ? 65536 / (NT * (PL::RM <= 16 ? 64 : 128)) : 1;
}
template <class PL>
__host__ __device__ constexpr int row_min_blocks() { return pass_min_blocks<PL, row_lines<PL>() * PL::TMAX>(); }
// plain row pass (READ = false); the readout planes use k_row_pass_read
template <class PL, bool READ>
__global__ void __launch_bounds__(row_lines<PL>() * PL::TMAX, row_min_blocks<PL>())
k_row_pass(const PassArgs p)
{
	row_pass_body<PL, READ>(p);
}
template <class PL>
__global__ void __launch_bounds__(row_lines<PL>() * PL::TMAX, read_min_blocks<PL>())
k_row_pass_read(const PassArgs p)
{
	row_pass_body<PL, true>(p);
}

// Live rows of a column-pass thread as a bit mask: bit m is set when row
// y = j + B m (m < A) lies outside the band gap (k1, k2), i.e. y <= k1 or
// y >= k2.  One mask per thread replaces a comparison per element.
template <int A, int B>
__device__ __forceinline__ unsigned live_rows(int j, int k1, int k2)
{
	static_assert(A <= 32, "one bit per value");
	const int lo = k1 >= j ? min((k1 - j) / B, A - 1) : -1;          // last m with y <= k1
	const int hi = k2 > j ? min((k2 - j + B - 1) / B, 32) : 0;       // first m with y >= k2
	const unsigned low = lo < 0 ? 0u : (lo >= 31 ? 0xffffffffu : ((2u << lo) - 1u));
	const unsigned high = hi >= 32 ? 0u : (0xffffffffu << hi);
	return low | high;
}

// Column pass: IFT_y -> real-space readout (plane) -> x t -> FT_y.  NXC is the
// row stride when it is known at compile time (square grids, nx = N), so the
// element offsets of the wave and grating accesses are constants; 0 reads it
// from the arguments.
// The pass on one tile (wave b, columns col0 ... col0 + C - 1).  SYNC places a
// CTA barrier between the wave loads and the first transform (which makes a
// shared twiddle copy filled just before visible).
template <class PL, bool READ, int NXC, bool SYNC, class TW>
__device__ __forceinline__ void col_pass_tile(const PassArgs& p, int b, int col0, const TW& tw, float2* sm)
{
	constexpr int C = PL::CC;
	using T = ColTile<C>;
	const int tid = threadIdx.x;
	const int nx = NXC > 0 ? NXC : p.nx;
	const int nval = min(C, nx - col0);
	float2* W = p.work + (long long)b * p.wstride + col0;
	float2 v[PL::RM];
	#pragma unroll
	for (int m = 0; m < PL::RM; m++) v[m] = make_float2(0.f, 0.f);
	int c, j;
	T::template role<PL::T>(tid, c, j);
	// 32-bit offsets within a wave (nx * ny < 2^31): one base pointer per
	// thread and a row stride, instead of a 64-bit product per element
	const int stride = PL::B * nx;
	if (c < nval && j < PL::T) {
		const float2* src = W + j * nx + c;
		const unsigned lin = live_rows<PL::A, PL::B>(j, p.in_k1, p.in_k2);
		#pragma unroll
		for (int m = 0; m < PL::A; m++)
			if (lin & (1u << m)) v[m] = src[m * stride];
	}
	if constexpr (SYNC) __syncthreads();
	PL::template to_mid<true, T>(v, sm, tw, tid);
	{
		int pos;
		T::template role<PL::TMID>(tid, c, pos);
		if (c < nval && pos < PL::TMID) {
			const int x = col0 + c;
			const float2* mul = p.mul + (p.mul_w ? __ldg(p.mul_w + b) : 0);   // this wave's grating
			if (p.npgx == nx && p.npgy == p.ny) { // grating of the grid size
				const float2* t = mul + x;
				#pragma unroll
				for (int e = 0; e < PL::EMID; e++) {
					const int y = PL::mid(pos, e);
					if (READ) readout_real(p, b, y, x, v[e]);
					v[e] = cmul(v[e], __ldg(t + y * nx));
				}
			}
			else { // sub-frame grating repeated periodically
				const int xs = x % p.npgx;
				#pragma unroll
				for (int e = 0; e < PL::EMID; e++) {
					const int y = PL::mid(pos, e);
					if (READ) readout_real(p, b, y, x, v[e]);
					v[e] = cmul(v[e], __ldg(mul + (long long)(y % p.npgy) * p.npgx + xs));
				}
			}
			int sx = p.plas_x, sy = p.plas_y;
			if (p.plas_w) { sx = __ldg(p.plas_w + 2 * b); sy = __ldg(p.plas_w + 2 * b + 1); }
			if (sx | sy) { // plasmon shift of the spectrum (uniform branch)
				const float tx = (float)(int)(((long long)sx * x) % nx) / (float)nx;
				#pragma unroll
				for (int e = 0; e < PL::EMID; e++) {
					const int y = PL::mid(pos, e);
					const float ty = (float)(int)(((long long)sy * y) % p.ny) / (float)p.ny;
					float sn, cs;
					sincospif(2.f * (tx + ty), &sn, &cs);
					v[e] = cmul(v[e], make_float2(cs, sn));
				}
			}
		}
	}
	PL::template from_mid<false, T>(v, sm, tw, tid);
	T::template role<PL::T>(tid, c, j);
	if (c < nval && j < PL::T) {
		float2* dst = W + j * nx + c;
		const unsigned lout = live_rows<PL::A, PL::B>(j, p.out_k1, p.out_k2);
		#pragma unroll
		for (int m = 0; m < PL::A; m++)
			if (lout & (1u << m)) dst[m * stride] = v[m];
	}
}

template <class PL, bool READ, int NXC>
__global__ void __launch_bounds__(PL::CC * PL::TMAX, PL::RM > 16 && !READ ? pass_min_blocks<PL, PL::CC * PL::TMAX>() : 0)
k_col_pass(const PassArgs p)
{
	extern __shared__ float2 sm[];
	__shared__ float2 tws[PL::TWS];
	if constexpr (PL::SMEM_TW) {
		fill_tw_shared<PL::A, PL::B, PL::CC * PL::TMAX>(tws, p.twy, threadIdx.x);   // barrier after the wave loads
		col_pass_tile<PL, READ, NXC, true>(p, blockIdx.y, blockIdx.x * PL::CC, TwShared<PL::B>{tws}, sm);
	}
	else col_pass_tile<PL, READ, NXC, false>(p, blockIdx.y, blockIdx.x * PL::CC, TwGlobal{p.twy}, sm);
}

// Exit column pass: IFT_y -> real-space readout (plane), no store.
template <class PL>
__global__ void __launch_bounds__(PL::CC * PL::TMAX)
k_exit_cols(const PassArgs p)
{
	constexpr int C = PL::CC;
	using T = ColTile<C>;
	extern __shared__ float2 sm[];
	const int tid = threadIdx.x, b = blockIdx.y, col0 = blockIdx.x * C;
	const int nval = min(C, p.nx - col0);
	const int nx = p.nx;
	const float2* W = p.work + (long long)b * p.wstride + col0;
	float2 v[PL::RM];
	#pragma unroll
	for (int m = 0; m < PL::RM; m++) v[m] = make_float2(0.f, 0.f);
	int c, j;
	T::template role<PL::T>(tid, c, j);
	if (c < nval && j < PL::T) {
		#pragma unroll
		for (int m = 0; m < PL::A; m++) {
			const int y = j + PL::B * m;
			if (y <= p.in_k1 || y >= p.in_k2) v[m] = W[(long long)y * nx + c];
		}
	}
	PL::template to_mid<true, T>(v, sm, TwGlobal{p.twy}, tid);
	int pos;
	T::template role<PL::TMID>(tid, c, pos);
	if (c < nval && pos < PL::TMID) {
		#pragma unroll
		for (int e = 0; e < PL::EMID; e++) readout_real(p, b, PL::mid(pos, e), col0 + c, v[e]);
	}
}

// ---------------------------------------------------------------------------
// launchers (explicitly instantiated per size in jms_inst_*.cu)
// ---------------------------------------------------------------------------
// closes a group of cp.async copies (the phase-grating synthesis stages its
// atom chunks with them)
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }

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

template <class PL>
int row_blocks_t(int ny) { return (ny + row_lines<PL>() - 1) / row_lines<PL>(); }

template <class PL>
cudaError_t launch_entry_t(const PassArgs& p, cudaStream_t s)
{
	constexpr int L = row_lines<PL>();
	constexpr int smem = PL::template smem_elems<RowTileOf<PL>>() * (int)sizeof(float2);
	return launch_k(k_entry_rows<PL>, dim3((p.ny + L - 1) / L, p.nwave), L * PL::TMAX, smem, p, s);
}
template <class PL>
cudaError_t launch_row_t(const PassArgs& p, cudaStream_t s)
{
	constexpr int L = row_lines<PL>();
	constexpr int smem = PL::template smem_elems<RowTileOf<PL>>() * (int)sizeof(float2);
	const dim3 grid((p.ny + L - 1) / L, p.nwave);
	if (p.plane >= 0) return launch_k(k_row_pass_read<PL>, grid, L * PL::TMAX, smem, p, s);
	return launch_k(k_row_pass<PL, false>, grid, L * PL::TMAX, smem, p, s);
}
template <class PL>
cudaError_t launch_col_t(const PassArgs& p, cudaStream_t s)
{
	constexpr int C = PL::CC;
	constexpr int smem = PL::template smem_elems<ColTile<C>>() * (int)sizeof(float2);
	const dim3 grid((p.nx + C - 1) / C, p.nwave);
	if (p.plane >= 0) {
		if (p.nx == PL::N) return launch_k(k_col_pass<PL, true, PL::N>, grid, C * PL::TMAX, smem, p, s);
		return launch_k(k_col_pass<PL, true, 0>, grid, C * PL::TMAX, smem, p, s);
	}
	if (p.nx == PL::N) return launch_k(k_col_pass<PL, false, PL::N>, grid, C * PL::TMAX, smem, p, s);
	return launch_k(k_col_pass<PL, false, 0>, grid, C * PL::TMAX, smem, p, s);
}
template <class PL>
cudaError_t launch_exit_t(const PassArgs& p, cudaStream_t s)
{
	constexpr int C = PL::CC;
	constexpr int smem = PL::template smem_elems<ColTile<C>>() * (int)sizeof(float2);
	return launch_k(k_exit_cols<PL>, dim3((p.nx + C - 1) / C, p.nwave), C * PL::TMAX, smem, p, s);
}

#define JMS_INSTANTIATE(PL) \
	template int row_blocks_t<PL>(int); \
	template cudaError_t launch_entry_t<PL>(const PassArgs&, cudaStream_t); \
	template cudaError_t launch_row_t<PL>(const PassArgs&, cudaStream_t); \
	template cudaError_t launch_col_t<PL>(const PassArgs&, cudaStream_t); \
	template cudaError_t launch_exit_t<PL>(const PassArgs&, cudaStream_t);

} // namespace jms
