/*
 * jms_oracle.cpp -- FP64 CPU restatement of JMultiSlice's multislice hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: tests/, the package's
 * smoke() and bench.py's CPU-baseline leg load it (through oracle/oracle.py)
 * to compare the CUDA product against it.  The product never links, loads or
 * calls anything here.
 *
 * What is restated (all arithmetic in double precision; inputs that the
 * reference holds in float -- gratings, propagators, detector functions,
 * the incident wave -- are taken as float and promoted):
 *   - the slice loop of CJMultiSlice::CPUMultislice        src/JMultiSlice.cpp:3589-3720
 *     (readout Fourier -> IFT -> readout real -> x t -> FT -> x P; exit readouts)
 *   - Fourier-space readout ReadoutDifDet_h               src/JMultiSlice.cpp:3369-3470
 *     with DotProduct_h / MaskedDotProduct_h sums          src/JMultiSlice.cpp:3279-3330
 *   - real-space readout ReadoutImgDet_h                  src/JMultiSlice.cpp:3473-3538
 *   - sub-frame grating multiply MultiplySub2dC           src/JFFTMKLcore.cpp:434-458
 *   - probe offset OffsetIncomingWave (CPU branch)        src/JMultiSlice.cpp:1999-2031
 *   - detection plane hash SetDetectionPlanes             src/JMultiSlice.cpp:579-626
 *   - variant draws GetRandomVariantSequence              src/JMultiSlice.cpp:1571-1676
 *   - plasmon Monte-Carlo shifts CJPlasmonMC::ScatGridMC  src/JPlasmonMC.cpp:153-209
 *     with CRng (std::mt19937 + uniform_int_distribution) src/rng.cpp:30-74
 *   - phase gratings of CJEElaSca (2-D projection mode)   src/JEElaSca.cpp:486-741, 812-976
 *     from radial form-factor tables (linear interpolation as
 *     CAtomType::GetFormFactor, src/Atoms.cpp:414-436)
 *   - unnormalised 2-D C2C transforms as MKL DFTI does    src/JFFTMKLcore.cpp:129-142,176,213
 *     (forward = exp(-i), backward = exp(+i), no scaling), here on a
 *     project-written mixed-radix FP64 FFT.
 */
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <cstdlib>
#include <random>
#include <thread>
#include <vector>

typedef std::complex<double> zd;

static const double kTwoPi = 6.283185307179586476925286766559;

// ---------------------------------------------------------------------------
// FP64 mixed-radix FFT (recursive decimation in time, any length).
// ---------------------------------------------------------------------------
namespace {

struct Plan {
	int n = 0;
	std::vector<int> fac;   // radices, product = n
	std::vector<zd> root;   // root[k] = exp(-2 pi i k / n), k < n
};

static void factorize(int n, std::vector<int>& f)
{
	f.clear();
	while (n % 4 == 0) { f.push_back(4); n /= 4; }
	while (n % 2 == 0) { f.push_back(2); n /= 2; }
	for (int p = 3; p * p <= n; p += 2)
		while (n % p == 0) { f.push_back(p); n /= p; }
	if (n > 1) f.push_back(n);
}

static void make_plan(Plan& P, int n)
{
	P.n = n;
	factorize(n, P.fac);
	P.root.resize(n);
	for (int k = 0; k < n; k++) {
		double a = -kTwoPi * (double)k / (double)n;
		P.root[k] = zd(std::cos(a), std::sin(a));
	}
}

static inline zd cmul(zd a, zd b)
{
	return zd(a.real() * b.real() - a.imag() * b.imag(), a.real() * b.imag() + a.imag() * b.real());
}

// out[0..n) = DFT of in[0], in[is], ..., sign -1 (forward) or +1 (backward).
// rstride maps this sub-transform's roots onto the plan's root table.
static void fft_rec(const Plan& P, zd* out, const zd* in, int n, long is, int fi, int rstride, int sign,
	std::vector<zd>& scratch)
{
	if (n == 1) { out[0] = in[0]; return; }
	const int p = P.fac[fi];
	const int m = n / p;
	for (int q = 0; q < p; q++)
		fft_rec(P, out + (long)q * m, in + (long)q * is, m, is * p, fi + 1, rstride * p, sign, scratch);
	zd t[64];
	zd* tp = (p <= 64) ? t : scratch.data();
	if (p > 64 && (int)scratch.size() < p) { scratch.resize(p); tp = scratch.data(); }
	for (int k = 0; k < m; k++) {
		for (int q = 0; q < p; q++) {
			long e = ((long)q * k * rstride) % P.n;
			zd w = P.root[e];
			if (sign > 0) w = std::conj(w);
			tp[q] = cmul(out[(long)q * m + k], w);
		}
		for (int r = 0; r < p; r++) {
			zd s(0.0, 0.0);
			for (int q = 0; q < p; q++) {
				long e = ((long)q * r % p) * (long)(P.n / p);
				zd w = P.root[e];
				if (sign > 0) w = std::conj(w);
				s += cmul(tp[q], w);
			}
			out[(long)r * m + k] = s;
		}
	}
}

static void fft1d(const Plan& P, zd* data, long stride, int sign, std::vector<zd>& buf, std::vector<zd>& scratch)
{
	const int n = P.n;
	buf.resize(2 * (size_t)n);
	zd* in = buf.data();
	zd* out = buf.data() + n;
	for (int i = 0; i < n; i++) in[i] = data[(long)i * stride];
	fft_rec(P, out, in, n, 1, 0, 1, sign, scratch);
	for (int i = 0; i < n; i++) data[(long)i * stride] = out[i];
}

// Runs body(i) for i in [0, n) on up to OR_THREADS host threads
// (default: all hardware threads).
template <class F>
static void parallel_for(int n, F body)
{
	int nt = (int)std::thread::hardware_concurrency();
	if (const char* e = std::getenv("OR_THREADS")) nt = std::atoi(e);
	if (nt < 1) nt = 1;
	if (nt > n) nt = n;
	if (nt <= 1 || n < 64) { for (int i = 0; i < n; i++) body(i); return; }
	std::vector<std::thread> pool;
	for (int t = 0; t < nt; t++)
		pool.emplace_back([=, &body]() { for (int i = t; i < n; i += nt) body(i); });
	for (auto& th : pool) th.join();
}

static void fft2d(zd* w, int nx, int ny, int sign)
{
	Plan px, py;
	make_plan(px, nx);
	make_plan(py, ny);
	parallel_for(ny, [&](int j) {
		thread_local std::vector<zd> buf, scratch;
		fft1d(px, w + (long)j * nx, 1, sign, buf, scratch);
	});
	parallel_for(nx, [&](int i) {
		thread_local std::vector<zd> buf, scratch;
		fft1d(py, w + i, nx, sign, buf, scratch);
	});
}

static inline int imod(int a, int b) { int r = a % b; return r >= 0 ? r : r + b; }

} // namespace

extern "C" {

// In-place unnormalised 2-D transform of an interleaved complex128 array
// [ny][nx]; sign -1 = forward (MKL DftiComputeForward), +1 = backward.
void or_fft2d(double* z, int nx, int ny, int sign)
{
	fft2d(reinterpret_cast<zd*>(z), nx, ny, sign);
}

// SetDetectionPlanes, period overload (src/JMultiSlice.cpp:579-626).
// det_objslc receives nobjslc+1 entries; returns the number of planes.
int or_detection_planes(int ndetper, int nobjslc, int* det_objslc)
{
	int ndetslc = 0;
	int noslc = nobjslc > 0 ? nobjslc : 0;
	if (det_objslc && nobjslc > 0)
		for (int i = 0; i <= nobjslc; i++) det_objslc[i] = -1;
	if (ndetper > 0) {
		if (noslc > 0) {
			for (int i = 0; i <= noslc; i++) {
				if (i % ndetper == 0) { if (det_objslc) det_objslc[i] = ndetslc; ndetslc++; }
			}
			if (noslc % ndetper != 0) { if (det_objslc) det_objslc[noslc] = ndetslc; ndetslc++; }
		}
		else { if (det_objslc) det_objslc[0] = 0; ndetslc = 1; }
	}
	else { if (det_objslc) det_objslc[noslc] = 0; ndetslc = 1; }
	return ndetslc;
}

// ---------------------------------------------------------------------------
// CRng restated (src/rng.cpp:30-74): mt19937 seeded with the int seed, draws
// uniform ints in [0, 0x7FFFFFFF]; unirand(a,b) = a + r/0x7FFFFFFF*(b-a).
// ---------------------------------------------------------------------------
struct OrRng {
	std::mt19937 urng;
	std::uniform_int_distribution<int> uni{0, 0x7FFFFFFF};
	double unirand(double a, double b)
	{
		return a + ((double)uni(urng) / (double)((unsigned long)0x7FFFFFFF)) * (b - a);
	}
};

void* or_rng_create(int seed) { OrRng* r = new OrRng(); r->urng.seed(seed); return r; }
void or_rng_destroy(void* r) { delete (OrRng*)r; }

// GetRandomVariantSequence (src/JMultiSlice.cpp:1571-1676): per object slice,
// draw a variant of its structure slice without replacement from a per-slice
// queue, never repeating the previous draw of that slice at a queue refill.
int or_variant_sequence(void* rng, int nscslc, const int* nvarslc, int nobjslc, const int* objslc, int* out)
{
	OrRng* R = (OrRng*)rng;
	if (!R || !out || !nvarslc || !objslc || nscslc < 1 || nobjslc < 1) return 2;
	int qmax = 0;
	for (int i = 0; i < nscslc; i++) qmax = nvarslc[i] > qmax ? nvarslc[i] : qmax;
	std::vector<int> q((size_t)nscslc * (qmax > 0 ? qmax : 1), 0), qlen(nscslc, 0), qlast(nscslc, -1);
	for (int i = 0; i < nobjslc; i++) {
		int s = objslc[i];
		int nv = nvarslc[s];
		if (nv < 2) { out[i] = 0; continue; }
		int* qc = &q[(size_t)s * qmax];
		if (qlen[s] <= 0) { for (int j = 0; j < nv; j++) qc[j] = j; qlen[s] = nv; }
		int k = (int)R->unirand(0.0, (double)nv);
		k = k % nv;
		int k0 = k;
		while (qc[k] < 0 || qc[k] == qlast[s]) {
			k = (k + 1) % nv;
			if (k == k0) break;
		}
		int v = qc[k];
		if (v < 0) { v = (int)R->unirand(0.0, (double)nv); qlen[s] = 0; }
		else { qc[k] = -1; qlen[s]--; }
		qlast[s] = v;
		out[i] = v;
	}
	return 0;
}

// Bulk plasmon Monte-Carlo path of one multislice run (CJPlasmonMC, src/JPlasmonMC.cpp:
// 153-209, as GPUMultislice / CPUMultislice draw it after the variant sequence,
// src/JMultiSlice.cpp:4583-4603, 3650-3690): per object slice j >= islc0 a
// Poisson number of new excitations (mean dt_j / mfp, float), capped at the
// remaining budget nexmax; each adds q (q^2 = qe^2 ((qc/qe)^2 + 1)^u - qe^2)
// in the direction 2 pi u'; the spectrum moves by the change of
// round(q_total * a) pixels.  shifts [nobjslc][2] (x, y pixels), zero where
// nothing moves.  The arithmetic is float as in the reference.
int or_plasmon_shifts(void* rng, int nobjslc, int islc0, const float* dt, float ax, float ay, float q_e,
	float q_c, float mfp, unsigned int nexmax, int* shifts)
{
	OrRng* R = (OrRng*)rng;
	if (!R || !shifts || !dt) return 2;
	for (int j = 0; j < 2 * nobjslc; j++) shifts[j] = 0;
	q_e = std::fabs(q_e); q_c = std::fabs(q_c); mfp = std::fabs(mfp);
	if (mfp <= 0.f || q_e <= 0.f || q_c < q_e) return 0;
	const float qe2 = q_e * q_e, qc2 = q_c * q_c;
	unsigned int nex = 0;
	float tqx = 0.f, tqy = 0.f;
	for (int j = (islc0 < 0 ? 0 : islc0); j < nobjslc; j++) {
		std::poisson_distribution<int> pd((double)(dt[j] / mfp));
		unsigned int n = (unsigned int)pd(R->urng);
		if (n > nexmax - nex) n = nexmax - nex;
		if (n == 0) continue;
		float qx = 0.f, qy = 0.f;
		for (unsigned int i = 0; i < n; i++) {
			const float phi = (float)(kTwoPi * R->unirand(0.0, 1.0));
			const float u = (float)R->unirand(0.0, 1.0);
			const float q = std::sqrt(qe2 * std::pow(qc2 / qe2 + 1.f, u) - qe2);
			qx += q * std::cos(phi);
			qy += q * std::sin(phi);
		}
		const int i0 = (int)std::round(tqx * ax), j0 = (int)std::round(tqy * ay);
		nex += n;
		tqx += qx;
		tqy += qy;
		shifts[2 * j] = (int)std::round(tqx * ax) - i0;
		shifts[2 * j + 1] = (int)std::round(tqy * ay) - j0;
	}
	return 0;
}

// OffsetIncomingWave, CPU branch (src/JMultiSlice.cpp:1999-2031), in FP64:
// out(k) = wav0(k - tilt) * exp(-i [2 pi (kx dx + ky dy + k^2 dz wl/2) + cppl(k)]).
// kx = fnx(i)/a, ky = fny(j)/b with the scrambled frequency numbers of
// InitCore (src/JMultiSlice.cpp:1710-1723).  cppl may be NULL.
void or_offset(int nx, int ny, double a, double b, double wl, const float* wav0, double dx, double dy,
	double dz, const float* cppl, int ibtx, int ibty, double* out)
{
	const std::complex<float>* w0 = reinterpret_cast<const std::complex<float>*>(wav0);
	zd* o = reinterpret_cast<zd*>(out);
	int nx2 = (nx - (nx % 2)) >> 1, ny2 = (ny - (ny % 2)) >> 1;
	double fz = dz * wl * 0.5;
	for (int j = 0; j < ny; j++) {
		double ky = (double)(((j + ny2) % ny) - ny2) / b;
		int js = imod(j - ibty, ny);
		for (int i = 0; i < nx; i++) {
			double kx = (double)(((i + nx2) % nx) - nx2) / a;
			long idx = (long)j * nx + i;
			double chi = kTwoPi * (ky * (dy + ky * fz) + kx * (dx + kx * fz)) + (cppl ? (double)cppl[idx] : 0.0);
			zd pp(std::cos(chi), -std::sin(chi));
			std::complex<float> s = w0[(long)js * nx + imod(i - ibtx, nx)];
			o[idx] = cmul(zd(s.real(), s.imag()), pp);
		}
	}
}

// One multislice run (CPUMultislice, src/JMultiSlice.cpp:3589-3720) in FP64.
//  wav      in/out complex128 [ny][nx], Fourier space on entry (offset applied)
//  pgr      complex64 grating pool [*][npgy][npgx]; pgr_idx[jslc] selects the
//           grating of object slice jslc (structure slice and variant resolved)
//  pro      complex64 propagator pool [*][ny][nx]; pro_idx[jslc] selects
//  det_objslc  [nobjslc+1] plane hash (-1 = no readout)
//  det      float [ndet][ny][nx]; msklen[idet] > 0 restricts the sum to the
//           msk entries (concatenated over detectors)
//  outputs are accumulated with weight (caller clears them for accmode 0):
//  det_int [ndetslc][ndet]; dif, img [ndetslc][N] (or NULL); wff, wfr complex
//  [ndetslc][N] (or NULL).  imagedet uses the _JMS_DETECT_* bits
//  (src/JMultiSlice.h:139-149).
int or_multislice(int nx, int ny, double* wav, int nobjslc, int islc0,
	const float* pgr, int npgx, int npgy, const int* pgr_idx,
	const float* pro, const int* pro_idx, const int* det_objslc,
	int ndet, const float* det, const int* msklen, const int* msk,
	int imagedet, double weight,
	double* det_int, double* dif, double* img, double* wff, double* wfr, const int* shifts)
{
	const long N = (long)nx * ny;
	zd* w = reinterpret_cast<zd*>(wav);
	const std::complex<float>* pg = reinterpret_cast<const std::complex<float>*>(pgr);
	const std::complex<float>* pr = reinterpret_cast<const std::complex<float>*>(pro);
	const bool b_img = (imagedet & (2 | 8 | 32 | 128)) != 0;
	const bool b_dif = (imagedet & (1 | 4 | 16 | 64 | 256)) != 0;
	std::vector<long> mskoff(ndet > 0 ? ndet : 1, 0);
	for (int d = 1; d < ndet; d++) mskoff[d] = mskoff[d - 1] + (msklen ? msklen[d - 1] : 0);

	auto readout_dif = [&](int islc) {
		int id = det_objslc[islc];
		if (id < 0) return;
		if ((imagedet & 1) && ndet > 0) {
			for (int d = 0; d < ndet; d++) {
				const float* D = det + (long)d * N;
				double s = 0.0;
				if (msklen && msklen[d] > 0) {
					const int* m = msk + mskoff[d];
					for (int t = 0; t < msklen[d]; t++) s += std::norm(w[m[t]]) * (double)D[m[t]];
				}
				else {
					for (long t = 0; t < N; t++) s += std::norm(w[t]) * (double)D[t];
				}
				det_int[(long)id * ndet + d] += weight * s;
			}
		}
		if (dif && (imagedet & (4 | 64))) for (long t = 0; t < N; t++) dif[(long)id * N + t] += weight * std::norm(w[t]);
		if (wff && (imagedet & (16 | 256))) {
			zd* o = reinterpret_cast<zd*>(wff) + (long)id * N;
			for (long t = 0; t < N; t++) o[t] += weight * w[t];
		}
	};
	auto readout_img = [&](int islc) {
		int id = det_objslc[islc];
		if (id < 0) return;
		if (img && (imagedet & (2 | 32))) for (long t = 0; t < N; t++) img[(long)id * N + t] += weight * std::norm(w[t]);
		if (wfr && (imagedet & (8 | 128))) {
			zd* o = reinterpret_cast<zd*>(wfr) + (long)id * N;
			for (long t = 0; t < N; t++) o[t] += weight * w[t];
		}
	};

	int islc = islc0 < 0 ? 0 : (islc0 > nobjslc ? nobjslc : islc0);
	for (int j = islc; j < nobjslc; j++) {
		if (b_dif) readout_dif(j);
		fft2d(w, nx, ny, +1);
		if (b_img) readout_img(j);
		const std::complex<float>* t = pg + (long)pgr_idx[j] * npgx * npgy;
		for (int y = 0; y < ny; y++) {
			for (int x = 0; x < nx; x++) {
				std::complex<float> tv = t[(long)(y % npgy) * npgx + (x % npgx)];
				long i = (long)y * nx + x;
				w[i] = cmul(w[i], zd(tv.real(), tv.imag()));
			}
		}
		fft2d(w, nx, ny, -1);
		if (shifts && (shifts[2 * j] || shifts[2 * j + 1])) { // plasmon: cyclic shift of the spectrum (CShift2d)
			std::vector<zd> t(w, w + N);
			const int sx = imod(shifts[2 * j], nx), sy = imod(shifts[2 * j + 1], ny);
			for (int y = 0; y < ny; y++)
				for (int x = 0; x < nx; x++)
					w[(long)((y + sy) % ny) * nx + (x + sx) % nx] = t[(long)y * nx + x];
		}
		const std::complex<float>* P = pr + (long)pro_idx[j] * N;
		for (long i = 0; i < N; i++) w[i] = cmul(w[i], zd(P[i].real(), P[i].imag()));
	}
	if (b_dif) readout_dif(nobjslc);
	if (b_img) {
		fft2d(w, nx, ny, +1);
		readout_img(nobjslc);
	}
	return 0;
}

// Phase grating of one structure slice, CJEElaSca::CalculatePhasegratingCPU
// (src/JEElaSca.cpp:812-976) in FP64:
//   pot(q) = sum_atoms occ ff_type(|q|) ap1(q)^2 exp(-2 pi i (fx fi + fy fj))
//            (ap1 = 0.5 - 0.5 tanh((|q| / kmax - 0.9) 30) if bwl_pot, else 1;
//             src/JEElaSca.cpp:597-600, applied in PrepareScatteringFunctions
//             :738-739 and again in the add :934)
//   V'(r)  = backward transform of pot (unscaled)
//   t      = exp(i c V'),  c = wl cz / (4 pi vol) with vol = a b cz: the
//            reference's POT_SCA / vol and PGR_SIG cz wl (:947, 956-963), whose
//            constant product is 1 / (4 pi)
//   bwl_pgr: t = backward[ forward[t] * ap2 ], ap2 = 1 / (nx ny) for
//            |q| <= 2/3 kmax, 0 beyond (:602-609, :965-969).
// atoms: [natom][2] fractional positions (x / a, y / b) as used (sites,
// displaced or not); occ [natom]; type [natom]; ff [ntype][nk] complex float.
int or_pgr(int nx, int ny, double a, double b, double wl, int natom, const double* pos, const float* occ,
           const int* type, int ntype, int nk, double sk, const float* ff, int bwl_pot, int bwl_pgr, double* out)
{
	const long N = (long)nx * ny;
	zd* t = reinterpret_cast<zd*>(out);
	const int nx2 = (nx - nx % 2) >> 1, ny2 = (ny - ny % 2) >> 1;
	const double kmax = std::min(nx2 / a, ny2 / b);
	std::vector<zd> ex((size_t)natom * nx), ey((size_t)natom * ny);
	for (int k = 0; k < natom; k++) {
		if (type[k] < 0 || type[k] >= ntype) return 2;
		for (int i = 0; i < nx; i++) {
			double tt = pos[2 * k] * (double)(imod(i + nx2, nx) - nx2);
			tt -= std::floor(tt);
			ex[(size_t)k * nx + i] = zd(std::cos(kTwoPi * tt), -std::sin(kTwoPi * tt));
		}
		for (int j = 0; j < ny; j++) {
			double tt = pos[2 * k + 1] * (double)(imod(j + ny2, ny) - ny2);
			tt -= std::floor(tt);
			ey[(size_t)k * ny + j] = zd(std::cos(kTwoPi * tt), -std::sin(kTwoPi * tt)) * (double)occ[k];
		}
	}
	auto qabs = [&](int i, int j) {
		const double qx = (imod(i + nx2, nx) - nx2) / a, qy = (imod(j + ny2, ny) - ny2) / b;
		return std::sqrt(qx * qx + qy * qy);
	};
	parallel_for(ny, [&](int j) {
		std::vector<zd> fq(ntype);
		for (int i = 0; i < nx; i++) {
			const double q = qabs(i, j);
			double ap = 1.0;
			if (bwl_pot) ap = 0.5 - 0.5 * std::tanh((q / kmax - 0.9) * 30.0);
			const double fp = q / sk;
			int i0 = (int)std::floor(fp);
			if (i0 > nk - 2) i0 = nk - 2;
			const double w1 = fp - i0;
			for (int ty = 0; ty < ntype; ty++) {
				const float* f = ff + 2 * ((long)ty * nk + i0);
				fq[ty] = zd(f[0] * (1 - w1) + f[2] * w1, f[1] * (1 - w1) + f[3] * w1) * (ap * ap);
			}
			zd acc(0, 0);
			for (int k = 0; k < natom; k++) acc += fq[type[k]] * ex[(size_t)k * nx + i] * ey[(size_t)k * ny + j];
			t[(long)j * nx + i] = acc;
		}
	});
	fft2d(t, nx, ny, +1);
	const double c = wl / (4.0 * std::acos(-1.0) * a * b);
	for (long i = 0; i < N; i++) {
		const double ph = c * t[i].real(), am = std::exp(-c * t[i].imag());
		t[i] = zd(am * std::cos(ph), am * std::sin(ph));
	}
	if (bwl_pgr) {
		fft2d(t, nx, ny, -1);
		const double kthr = kmax * 2.0 / 3.0;
		for (int j = 0; j < ny; j++)
			for (int i = 0; i < nx; i++)
				t[(long)j * nx + i] *= (qabs(i, j) > kthr) ? 0.0 : 1.0 / (double)N;
		fft2d(t, nx, ny, +1);
	}
	return 0;
}

} // extern "C"
