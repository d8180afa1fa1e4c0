// jms_fft.cuh -- register/shared-memory FFT building blocks for sm_100a.
//
// The multislice step needs unnormalised 2-D C2C transforms of the wave
// (forward = exp(-i), inverse = exp(+i), no scaling), as the reference takes
// them from cuFFT (src/JFFTCUDAcore.cpp:299-336) and MKL
// (src/JFFTMKLcore.cpp:170-241).  Here every 1-D line transform of length
// N = A*B is done in two register stages with one shared-memory exchange:
//
//   stage 1: thread j (0 <= j < B) holds x[j + B*m], m < A; it runs an
//            A-point DFT in registers and multiplies by W_N^(j*k1);
//   exchange through shared memory;
//   stage 2: thread k1 (0 <= k1 < A) holds the B values of row k1 and runs a
//            B-point DFT; it ends up with X[k1 + A*k2], k2 < B.
//
// Both the loads before stage 1 (stride-B elements per thread, consecutive
// threads on consecutive elements) and the stores after stage 2 are
// coalesced, so a line never needs a staging pass through shared memory.
// A forward transform with (A,B) leaves data in exactly the layout an inverse
// transform with (B,A) expects, which lets one kernel run FT -> x P -> IFT
// (or IFT -> x t -> FT) on a line without touching global memory in between.
//
// In-register DFTs are mixed radix (2, 3, 4, 5) with compile-time twiddles:
// every index is a template constant (static_for), so the twiddles are literal
// constants computed in double by constexpr trigonometry and rounded once.
#pragma once
#include <cuda_runtime.h>
#include <utility>

namespace jms {

// ---------------------------------------------------------------------------
// compile-time loops and trigonometry
// ---------------------------------------------------------------------------
template <int... Is, class F>
__device__ __forceinline__ void static_for_impl(std::integer_sequence<int, Is...>, F&& f)
{
	(f(std::integral_constant<int, Is>{}), ...);
}
template <int N, class F>
__device__ __forceinline__ void static_for(F&& f)
{
	static_for_impl(std::make_integer_sequence<int, N>{}, f);
}

constexpr double kPi = 3.14159265358979323846264338327950288;

// sin and cos of x for |x| <= pi/4 by Taylor series (exact to double rounding)
__host__ __device__ constexpr double cx_sin_small(double x)
{
	double t = x, s = x;
	for (int k = 1; k < 14; k++) { t *= -x * x / ((2.0 * k) * (2.0 * k + 1.0)); s += t; }
	return s;
}
__host__ __device__ constexpr double cx_cos_small(double x)
{
	double t = 1.0, s = 1.0;
	for (int k = 1; k < 14; k++) { t *= -x * x / ((2.0 * k - 1.0) * (2.0 * k)); s += t; }
	return s;
}
// cos / sin of 2*pi*num/den with exact octant reduction in integers
__host__ __device__ constexpr double cx_cos_turn(long num, long den)
{
	num %= den; if (num < 0) num += den;
	// angle = 2 pi num/den; work in units of den/8 (octants)
	long n8 = num * 8;
	long oct = n8 / den;                 // octant 0..7
	double frac = (double)(n8 - oct * den) / (double)den; // in [0,1) of an octant
	double x = frac * (kPi / 4.0);
	double c = 0, s = 0;
	switch (oct) {
	case 0: c = cx_cos_small(x); break;
	case 1: c = cx_sin_small(kPi / 4.0 - x); break;
	case 2: c = -cx_sin_small(x); break;
	case 3: c = -cx_cos_small(kPi / 4.0 - x); break;
	case 4: c = -cx_cos_small(x); break;
	case 5: c = -cx_sin_small(kPi / 4.0 - x); break;
	case 6: c = cx_sin_small(x); break;
	default: c = cx_cos_small(kPi / 4.0 - x); break;
	}
	(void)s;
	return c;
}
__host__ __device__ constexpr double cx_sin_turn(long num, long den)
{
	// sin(2 pi num/den) = cos(2 pi (num/den - 1/4)) = cos(2 pi (4 num - den) / (4 den))
	return cx_cos_turn(4 * num - den, 4 * den);
}

// ---------------------------------------------------------------------------
// complex helpers
// ---------------------------------------------------------------------------
// Complex add and subtract as one packed FP32x2 instruction each (sm_100:
// add.f32x2 / fma.f32x2, both lanes rounded to nearest like the scalar
// forms).  a - b is formed as fma(b, -1, a): b * -1 is exact, so the result is
// the correctly rounded difference.
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b)
{
	return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) // a * conj(b)
{
	return make_float2(fmaf(a.x, b.x, a.y * b.y), fmaf(a.y, b.x, -a.x * b.y));
}
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
__device__ __forceinline__ float cnorm(float2 a) { return fmaf(a.x, a.x, a.y * a.y); }

// multiply by exp(sgn * 2 pi i E / R) with compile-time E, R; sgn = -1 for the
// forward transform, +1 for the inverse.  Trivial angles cost no multiply.
template <int E, int R, bool INV>
__device__ __forceinline__ float2 twiddle_ct(float2 v)
{
	constexpr int e = ((E % R) + R) % R;
	if constexpr (e == 0) {
		return v;
	}
	else if constexpr (4 * e == R) { // angle -+pi/2: forward multiplies by -i
		return INV ? make_float2(-v.y, v.x) : make_float2(v.y, -v.x);
	}
	else if constexpr (2 * e == R) {
		return make_float2(-v.x, -v.y);
	}
	else if constexpr (4 * e == 3 * R) {
		return INV ? make_float2(v.y, -v.x) : make_float2(-v.y, v.x);
	}
	else {
		constexpr float c = (float)cx_cos_turn(e, R);
		constexpr float s = INV ? (float)cx_sin_turn(e, R) : -(float)cx_sin_turn(e, R);
		return make_float2(fmaf(v.x, c, -v.y * s), fmaf(v.x, s, v.y * c));
	}
}

__host__ __device__ constexpr int first_factor(int r)
{
	return (r % 4 == 0) ? 4 : (r % 2 == 0) ? 2 : (r % 3 == 0) ? 3 : (r % 5 == 0) ? 5 : r;
}

// In-register DFT of x[OFF + S*i], i < R (natural order in and out).
template <int R, int S, int OFF, bool INV, int LEN>
__device__ __forceinline__ void dft_reg(float2 (&x)[LEN])
{
	if constexpr (R == 1) {
		return;
	}
	else if constexpr (R == 2) {
		float2 a = x[OFF], b = x[OFF + S];
		x[OFF] = cadd(a, b);
		x[OFF + S] = csub(a, b);
	}
	else if constexpr (R == 4) {
		float2 a = x[OFF], b = x[OFF + S], c = x[OFF + 2 * S], d = x[OFF + 3 * S];
		float2 t0 = cadd(a, c), t1 = csub(a, c), t2 = cadd(b, d), t3 = twiddle_ct<1, 4, INV>(csub(b, d));
		x[OFF] = cadd(t0, t2);
		x[OFF + 2 * S] = csub(t0, t2);
		x[OFF + S] = cadd(t1, t3);
		x[OFF + 3 * S] = csub(t1, t3);
	}
	else if constexpr (first_factor(R) == R) {
		// small odd prime: direct DFT with constant twiddles
		float2 in[R];
		static_for<R>([&](auto Q) { in[Q.value] = x[OFF + S * Q.value]; });
		static_for<R>([&](auto K) {
			constexpr int k = K.value;
			float2 s = in[0];
			static_for<R - 1>([&](auto Q) {
				constexpr int q = Q.value + 1;
				s = cadd(s, twiddle_ct<q * k, R, INV>(in[q]));
			});
			x[OFF + S * k] = s;
		});
	}
	else {
		// decimation in time: R = P * M; sub-DFTs on the P interleaved
		// sequences, twiddle W_R^(q k), then P-point DFTs across them.
		constexpr int P = first_factor(R);
		constexpr int M = R / P;
		float2 t[R];
		// t[q*M + i] = x[OFF + S*(q + P*i)]
		static_for<P>([&](auto Q) {
			static_for<M>([&](auto I) { t[Q.value * M + I.value] = x[OFF + S * (Q.value + P * I.value)]; });
		});
		static_for<P>([&](auto Q) { dft_reg<M, 1, Q.value * M, INV>(t); });
		static_for<M>([&](auto K) {
			constexpr int k = K.value;
			float2 u[P];
			static_for<P>([&](auto Q) {
				constexpr int q = Q.value;
				u[q] = twiddle_ct<q * k, R, INV>(t[q * M + k]);
			});
			dft_reg<P, 1, 0, INV>(u);
			static_for<P>([&](auto Q) { x[OFF + S * (k + M * Q.value)] = u[Q.value]; });
		});
	}
}

} // namespace jms
