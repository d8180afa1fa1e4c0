// jms_generators.cpp -- host-side setup generators of the multislice path.
//
// These produce the inputs of the hot path exactly as the reference does, so
// a caller switching libraries gets identical probes, propagators and
// detector functions (bit-identical on the same compiler / libm; the golden
// tests check them against the reference):
//   wavelength               src/JMultiSlice.cpp:372-378, constants src/NatureConstants.h
//   propagators (0 planar, 1 Fresnel, 2/3 band limit, 1/N scale)
//                            src/JMultiSlice.cpp:998-1106
//   ring detectors + masks   src/JMultiSlice.cpp:1274-1438 (+ profile file 1164-1272)
//   probe wave (aperture, aberrations, norm)
//                            src/JProbeGen.cpp:471-570, 707-776
//   detection planes         src/JMultiSlice.cpp:579-665
// The float / double mix of every expression follows the reference, because
// the values must agree to the last bit; the code itself is organised anew.
#include "jms_host.h"

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <fstream>

namespace jms {

// CODATA 2018 (SI)
static constexpr double kC0 = 299792458.;          // speed of light [m/s]
static constexpr double kHPL = 6.62607015E-34;     // Planck constant [J s]
static constexpr double kQEL = 1.602176634E-19;    // elementary charge [C]
static constexpr double kME0 = 9.1093837015E-31;   // electron rest mass [kg]
static constexpr double kPI = 3.1415926535897932384626433832795;
static constexpr double kTPI = 6.283185307179586476925286766559;
static constexpr double kRelAperture = 0.666666666666667; // band limit (fraction of Nyquist)

float wavelength_nm(float ht)
{
	// lambda [nm] = h c / e * 1e6 [nm keV] / sqrt(E (E + 2 m0 c^2)), E in keV
	const double two_e0_kev = 2. * kME0 * kC0 * kC0 / kQEL / 1000.;
	return (float)(kC0 * kHPL / kQEL * 1.0E+6 / std::sqrt(ht * (ht + two_e0_kev)));
}

float JmsB200::SetHighTension(float ht)
{
	const float old = ht_;
	ht_ = ht;
	wl_ = wavelength_nm(ht);
	return old;
}

// ---------------------------------------------------------------------------
// detection planes
// ---------------------------------------------------------------------------
int JmsB200::SetDetectionPlanes(int ndetper, int nobjslc, int* det_objslc) const
{
	const int nslc = std::max(0, nobjslc);
	if (det_objslc && nobjslc > 0) std::fill(det_objslc, det_objslc + nobjslc + 1, -1);
	int count = 0;
	auto mark = [&](int plane) { if (det_objslc) det_objslc[plane] = count; count++; };
	if (ndetper <= 0) {                 // exit plane only
		if (det_objslc) det_objslc[nslc] = 0;
		return 1;
	}
	if (nslc == 0) {                    // entrance plane only
		if (det_objslc) det_objslc[0] = 0;
		return 1;
	}
	for (int p = 0; p <= nslc; p += ndetper) mark(p); // entrance and periodic planes
	if (nslc % ndetper != 0) mark(nslc);               // out-of-period exit plane
	return count;
}

int JmsB200::SetDetectionPlanesList(const int* slc_det, int nlist, int nobjslc, int* det_objslc) const
{
	const int nslc = std::min(std::max(0, nobjslc), nlist);
	if (det_objslc && nobjslc > 0) std::fill(det_objslc, det_objslc + nobjslc + 1, -1);
	if (nlist <= 0) {
		if (det_objslc) det_objslc[nobjslc] = 0;
		return 1;
	}
	if (nslc == 0) {
		if (det_objslc) det_objslc[0] = 0;
		return 1;
	}
	int count = 0;
	for (int p = 0; p <= nslc; p++) {
		if (slc_det[p] >= 0) {
			if (det_objslc) det_objslc[p] = slc_det[p];
			count++;
		}
	}
	return count;
}

// ---------------------------------------------------------------------------
// propagator
// ---------------------------------------------------------------------------
static inline int scrambled_freq(int i, int n)
{
	const int nyq = (n - (n % 2)) >> 1;
	return ((i + nyq) % n) - nyq;
}

int JmsB200::CalculatePropagator(float fthick, float otx, float oty, float* pro_out, int ntype)
{
	if (pro_out == nullptr || ntype < 0 || ntype > 1) return 1;
	std::complex<float>* pro = reinterpret_cast<std::complex<float>*>(pro_out);
	const int nx = nx_, ny = ny_;
	const double sx = 1. / a0_[0], sy = 1. / a0_[1];   // Fourier sampling [1/nm]
	const int nyqx = (nx - (nx % 2)) >> 1, nyqy = (ny - (ny % 2)) >> 1;
	const double glim = std::min(sx * nyqx, sy * nyqy) * kRelAperture;
	const double glim2 = glim * glim;
	const double tx = (double)otx * (kPI / 180.), ty = (double)oty * (kPI / 180.);
	const double lam = (double)wl_;
	const double tilt = std::sqrt(tx * tx + ty * ty);
	const float amp = 1.f / ((float)nx * ny);           // keeps the norm over IFT / FT
	auto put = [&](long idx, double chi) {
		pro[idx] = std::complex<float>((float)std::cos(chi) * amp, (float)(-std::sin(chi) * amp));
	};
	if (ntype == 0) {
		// planar: exact path difference of a plane wave tilted by theta(g)
		nprotype_ = 0;
		const double k2pi = 2. * kPI / lam;
		const double ct = std::cos(tilt), st = std::sin(tilt);
		const double tdir = tilt > 0.0 ? std::atan2(ty, tx) : 0.;
		for (int j = 0; j < ny; j++) {
			const double gy = sy * scrambled_freq(j, ny);
			const double gy2 = gy * gy;
			for (int i = 0; i < nx; i++) {
				const double gx = sx * scrambled_freq(i, nx);
				const double g2 = gx * gx + gy2;
				const long idx = (long)j * nx + i;
				if (g2 > glim2) { pro[idx] = 0.f; continue; }
				const double th = std::asin(lam * std::sqrt(g2));
				const double az = th > 0. ? std::atan2(gy, gx) : 0.;
				const double path = 1. / (ct * std::cos(th) + st * std::sin(th) * std::cos(tdir - az)) - 1. / ct;
				put(idx, k2pi * (double)fthick * path);
			}
		}
	}
	else {
		// Fresnel: chi = dz pi/lambda cos(tilt) (|w - t|^2 - |t|^2)
		nprotype_ = 1;
		const double c = kPI / lam * std::cos(tilt);
		const double c0 = c * (tx * tx + ty * ty);
		const double wsx = sx * lam, wsy = sy * lam;
		const double wlim2 = glim2 * lam * lam;
		for (int j = 0; j < ny; j++) {
			const double wy = wsy * scrambled_freq(j, ny);
			const double wy2 = wy * wy;
			const double uy = wy - ty;
			const double uy2 = uy * uy;
			for (int i = 0; i < nx; i++) {
				const double wx = wsx * scrambled_freq(i, nx);
				const double w2 = wx * wx + wy2;
				const double ux = wx - tx;
				const double u2 = ux * ux + uy2;
				const long idx = (long)j * nx + i;
				if (w2 > wlim2) { pro[idx] = 0.f; continue; }
				put(idx, (double)fthick * (c * u2 - c0));
			}
		}
	}
	return 0;
}

// ---------------------------------------------------------------------------
// ring detector
// ---------------------------------------------------------------------------
// Sensitivity profile file: first line "<len> <refpix>", then one value per line
// (format of src/JMultiSlice.cpp:1164-1240).
static int load_profile(const char* path, std::vector<float>& prof, float& refpix)
{
	prof.clear();
	refpix = 0.f;
	std::ifstream in(path);
	if (!in.is_open()) return 1;
	std::string line;
	int len = 0;
	if (!std::getline(in, line)) return 2;
	{
		const std::string sep = "' ";
		size_t i0 = line.find_first_not_of(sep, 0);
		size_t i1 = line.find_first_of(sep, i0);
		if (i0 == std::string::npos || i1 == std::string::npos || i0 >= i1) return 2;
		len = std::stoi(line.substr(i0, i1 - i0));
		if (len > 0) {
			i0 = line.find_first_not_of(sep, i1);
			i1 = line.find_first_of(sep, i0);
			if (i1 == std::string::npos) i1 = line.length();
			if (i0 == std::string::npos || i0 >= i1) return 3;
			refpix = std::stof(line.substr(i0, i1 - i0));
		}
	}
	if (len <= 0) return 2;
	prof.assign((size_t)len + 10, 0.f);
	size_t k = 0;
	while (k < prof.size() && std::getline(in, line)) prof[k++] = std::stof(line);
	return 0;
}

static float radial_sensitivity(float theta, const std::vector<float>& prof, int len, float refpix, float beta1)
{
	// linear interpolation on a profile whose first sample is theta = 0 and whose
	// sample refpix (counted from 1) is at beta1
	const float rpix = std::max(0.f, refpix - 1.f);
	if (len <= 0 || rpix < 0.f) return 1.f;
	const float tpix = std::max(0.f, theta * rpix / beta1);
	const int ipix = (int)tpix;
	const float tfrac = tpix - ipix;
	if (ipix > len - 2) return prof[len - 1];
	return (1.f - tfrac) * prof[ipix] + tfrac * prof[ipix + 1];
}

int JmsB200::CalculateRingDetector(float beta0, float beta1, float phi0, float phi1, float theta0x, float theta0y,
	const char* sdsprofile, float* det, int* msklen, int* msk, int kmom1) const
{
	if (det == nullptr || msklen == nullptr) return 1;
	const int nx = nx_, ny = ny_;
	const long n = (long)nx * ny;
	*msklen = 0;
	std::fill(det, det + n, 0.f);
	if (msk) std::fill(msk, msk + n, 0);
	std::vector<float> prof;
	float refpix = 0.f;
	bool use_prof = false;
	if (sdsprofile && sdsprofile[0]) use_prof = (load_profile(sdsprofile, prof, refpix) == 0);
	const int proflen = use_prof ? (int)prof.size() - 10 : 0;
	const double sx = 1. / a0_[0], sy = 1. / a0_[1];
	const double k0 = 1. / (double)wl_;
	double r1 = (double)beta0 * 0.001, r2 = (double)beta1 * 0.001;
	double a1 = (double)phi0 * (kPI / 180.), a2 = (double)phi1 * (kPI / 180.);
	const double c1 = (double)theta0x * 0.001, c2 = (double)theta0y * 0.001;
	double gcx = 0., gcy = 0.;                       // detector centre [1/nm]
	if (nprotype_ == 1) {
		// small-angle mapping; the centre offset stays zero (reference behaviour)
		r1 *= k0;
		r2 *= k0;
	}
	else {
		r1 = k0 * std::sin(r1);
		r2 = k0 * std::sin(r2);
		const double gc = k0 * std::sin(std::sqrt(c1 * c1 + c2 * c2));
		const double az = gc > 0. ? std::atan2(c2, c1) : 0.;
		gcx = gc * std::cos(az);
		gcy = gc * std::sin(az);
	}
	const bool full_ring = (std::fabs(a1 - a2) < 0.0001) || (std::fabs(std::fabs(a1 - a2) - kTPI) < 0.0001);
	if (!full_ring) {
		while (a1 < 0.0 || a2 < 0.0) { a1 += kTPI; a2 += kTPI; }
		if (a1 >= a2) a2 += kTPI;
		while (a1 >= kTPI) { a1 -= kTPI; a2 -= kTPI; }
	}
	int count = 0;
	for (int j = 0; j < ny; j++) {
		const double gy = sy * scrambled_freq(j, ny) - gcy;
		const double gy2 = gy * gy;
		for (int i = 0; i < nx; i++) {
			const double gx = sx * scrambled_freq(i, nx) - gcx;
			const double g = std::sqrt(gy2 + gx * gx);
			double az = g > 0. ? std::atan2(gy, gx) : 0.;
			if (g < r1 || g >= r2) continue;
			if (!full_ring) {
				while (az < a1) az += kTPI;
				if (az < a1 || az >= a2) continue;
			}
			float s = 1.f;
			if (use_prof) {
				if (r1 > 0.) s = radial_sensitivity((float)g, prof, proflen, refpix, (float)r1);
				else if (r2 > 0.) s = radial_sensitivity((float)g, prof, proflen, refpix, (float)r2);
			}
			if (kmom1 == 1) s = s * (float)gx;
			else if (kmom1 == 2) s = s * (float)gy;
			const long idx = (long)j * nx + i;
			det[idx] = s;
			if (msk) msk[count++] = (int)idx;
		}
	}
	*msklen = msk ? count : 0;
	return 0;
}

// ---------------------------------------------------------------------------
// probe wave function
// ---------------------------------------------------------------------------
namespace {

// Axial aberration table of CJProbeGen (src/JProbeGen.cpp:178-214): 24 terms
// (order m = 1..8, rotational symmetry n = m, m-2, ... >= 0, listed with n
// ascending), binomial coefficients C(n, l).
struct AberrationTable {
	int order[24], sym[24];
	int binom[17][17];
	AberrationTable()
	{
		int l = 0;
		for (int m = 1; m <= 8; m++)
			for (int n = 0; n <= m; n++)
				if ((m + n) % 2 == 0) { order[l] = m; sym[l] = n; l++; }
		for (int n = 0; n < 17; n++)
			for (int k = 0; k < 17; k++) {
				if (k > n) { binom[n][k] = 0; continue; }
				int r = 1, kk = std::min(k, n - k);
				for (int i = 0; i < kk; i++) { r *= (n - i); r /= (i + 1); }
				binom[n][k] = r;
			}
	}
};
const AberrationTable kAbr;

// chi(q) [rad] of the coherent axial aberrations (src/JProbeGen.cpp:507-570)
float aberration_phase(float qx, float qy, float wl, const float* coeff)
{
	const float wx = qx * wl, wy = qy * wl;
	const float w = sqrtf(wx * wx + wy * wy);
	const float prefac = (float)kTPI / wl;
	float px[9], py[9], pa[9];
	px[0] = py[0] = pa[0] = 1.f;
	for (int i = 1; i < 9; i++) { px[i] = px[i - 1] * wx; py[i] = py[i - 1] * wy; pa[i] = pa[i - 1] * w; }
	static const float sgn[4] = {1.f, 0.f, -1.f, 0.f};
	float chi = 0.f;
	for (int k = 0; k < 24; k++) {
		const float cx = coeff[2 * k], cy = coeff[2 * k + 1];
		if (!((cx * cx + cy * cy) > (float)(1.E-15))) continue;
		const int m = kAbr.order[k], n = kAbr.sym[k];
		float term = 0.f;
		for (int l = 0; l <= n; l++) {
			float c = 0.f;
			c = c + sgn[l % 4] * cx;
			c = c + sgn[(l + 3) % 4] * cy;
			term = term + c * (float)kAbr.binom[n][l] * px[n - l] * py[l];
		}
		term = term * pa[m - n] / ((float)m);
		chi = chi + term;
	}
	return chi * prefac;
}

// smooth-edged, optionally distorted aperture (src/JProbeGen.cpp:471-504)
float aperture_amp(float qx, float qy, float qcx, float qcy, float qlim, float alim, float adir, float smooth)
{
	if (!(qlim > 0.f)) return 0.f;
	const float a1x = alim * cosf(2.f * adir);
	const float a1y = alim * sinf(2.f * adir);
	const float adet = 1.f - alim * alim;
	if (adet == 0.f) return 0.f;
	const float radet = 1.f / adet;
	const float dqx = qx - qcx, dqy = qy - qcy;
	const float ux = ((1.f - a1x) * dqx - a1y * dqy) * radet;
	const float uy = (-a1y * dqx + (1.f + a1x) * dqy) * radet;
	const float dq = sqrtf(ux * ux + uy * uy);
	const float edge = fabsf(smooth * qlim);
	if (!(dq > 0.f)) return 1.f;
	if (edge > 0.f) return (1.f - tanhf((float)kPI * (dq - qlim) / edge)) * 0.5f;
	return dq < qlim ? 1.f : 0.f;
}

} // namespace

int JmsB200::CalculateProbeWaveFourier(const ProbeParams& prm, float* wav_out) const
{
	if (wav_out == nullptr) return 1;
	if (wl_ <= 0.f || a0_[0] * a0_[1] <= 0.f || nx_ * ny_ <= 0 || prm.alpha <= 0.f) return 1;
	std::complex<float>* wav = reinterpret_cast<std::complex<float>*>(wav_out);
	const int nx = nx_, ny = ny_;
	const float wl = wl_;
	const float qlim = prm.alpha * 0.001f / wl;
	const float qcx = prm.alpha_x0 * 0.001f / wl, qcy = prm.alpha_y0 * 0.001f / wl;
	const float btx = prm.btx * 0.001f / wl, bty = prm.bty * 0.001f / wl;
	const float adir = prm.alpha_adir * 0.0174533f;
	std::vector<float> qx(nx), qy(ny);
	for (int i = 0; i < nx; i++) qx[i] = (float)scrambled_freq(i, nx) / a0_[0];
	for (int j = 0; j < ny; j++) qy[j] = (float)scrambled_freq(j, ny) / a0_[1];
	std::fill(wav, wav + (long)nx * ny, std::complex<float>(0.f, 0.f));
	float power = 0.f;
	for (int j = 0; j < ny; j++) {
		for (int i = 0; i < nx; i++) {
			const float amp = aperture_amp(qx[i] - btx, qy[j] - bty, qcx, qcy, qlim, prm.alpha_asym, adir, prm.alpha_rs);
			if (!(amp > (float)(1.E-6))) continue;
			const float chi = aberration_phase(qx[i], qy[j], wl, prm.abrr);
			wav[(long)j * nx + i] = std::complex<float>(amp * cosf(chi), -amp * sinf(chi));
			power += amp * amp;
		}
	}
	const float norm = 1.f / sqrtf(power);
	for (long k = 0; k < (long)nx * ny; k++) wav[k] = wav[k] * norm;
	return 0;
}

} // namespace jms
