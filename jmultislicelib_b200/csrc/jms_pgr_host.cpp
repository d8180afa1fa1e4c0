// jms_pgr_host.cpp -- host side of the on-device phase-grating generator.
//
// Follows the call sequence of CJEElaSca (src/JEElaSca.h:98-273):
// SetGrid / SetPhysics (grid, cell, beam energy, thermal model, band
// limits), the radial form-factor tables of the atom types (what
// CAtomType::CalculateRadialFormFactors prepares, src/Atoms.cpp:260-318, and
// CAtomType::CopyFormFactors hands out), then CalculatePhasegratingGPU
// (src/JEElaSca.cpp:978-1159) for a structure slice.  Differences, by design:
// many gratings per call (each with its own draw of the site displacements
// under the QEP model), results written straight into the multislice
// library's grating store, translation phases formed in FP64.
#include "jms_pgr_host.h"
#include "jms_kernels.h"
#include "jms_pgr.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

namespace jms {

namespace {
constexpr double kC0 = 299792458.;          // speed of light [m/s]
constexpr double kHPL = 6.62607015E-34;     // Planck constant [J s]
constexpr double kQEL = 1.602176634E-19;    // elementary charge [C]
constexpr double kME0 = 9.1093837015E-31;   // electron rest mass [kg]
constexpr double kPi = 3.141592653589793238462643383279502884;
constexpr float kSiteClose = 0.05f;         // atoms closer than this [nm] share a site (CStructure::SetAtomSites)

void dfree(void* p) { if (p) cudaFree(p); }

template <class T>
int dput(T*& d, size_t& cap, const T* h, size_t n, cudaStream_t s)
{
	if (n == 0) return 0;
	if (n > cap) {
		dfree(d);
		d = nullptr;
		cap = 0;
		if (cudaMalloc(&d, sizeof(T) * n) != cudaSuccess) return 4;
		cap = n;
	}
	if (h && cudaMemcpyAsync(d, h, sizeof(T) * n, cudaMemcpyHostToDevice, s) != cudaSuccess) return 5;
	return 0;
}

void twiddles(std::vector<float2>& tw, int n)
{
	tw.resize(n);
	for (int k = 0; k < n; k++) {
		const double ang = 2.0 * kPi * (double)k / (double)n;
		tw[k] = make_float2((float)std::cos(ang), (float)(-std::sin(ang)));
	}
}
} // namespace

PgrGen::~PgrGen() { Reset(); }

void PgrGen::SiteSet::release()
{
	dfree(base); dfree(ux); dfree(uy); dfree(asite); dfree(aocc); dfree(tstart);
	base = nullptr; ux = uy = nullptr; asite = tstart = nullptr; aocc = nullptr;
	key.clear();
}

void PgrGen::ClearSites()
{
	if (!sets_.empty() && stream_) cudaStreamSynchronize(stream_);
	for (SiteSet& t : sets_) t.release();
	sets_.clear();
}

void PgrGen::Reset()
{
	ClearSites();
	dfree(d_ff_); dfree(d_twx_); dfree(d_twy_); dfree(d_ap2_); dfree(d_buf_); dfree(d_out_); dfree(d_pos_);
	dfree(d_fq_); dfree(d_tab_);
	d_ff_ = nullptr; d_twx_ = d_twy_ = d_ap2_ = d_buf_ = d_out_ = nullptr;
	d_pos_ = nullptr;
	d_fq_ = d_tab_ = nullptr;
	fq_valid_ = false;
	cap_buf_ = cap_out_ = cap_pos_ = cap_tab_ = 0;
	status_ = 0;
	nx_ = ny_ = 0;
	ntype_ = nk_ = 0;
	biso_.clear();
}

int PgrGen::SetGrid(int nx, int ny, float a, float b)
{
	if (nx < 1 || ny < 1 || !(a > 0.f) || !(b > 0.f)) return 1;
	if (!pgr_supported(nx, ny)) return 8;
	ClearSites();
	dfree(d_twx_); dfree(d_twy_); dfree(d_ap2_);
	d_twx_ = d_twy_ = d_ap2_ = nullptr;
	fq_valid_ = false;
	nx_ = nx; ny_ = ny; a_ = a; b_ = b;
	std::vector<float2> tw;
	twiddles(tw, nx);
	if (cudaMalloc(&d_twx_, sizeof(float2) * nx) != cudaSuccess) return 4;
	cudaMemcpy(d_twx_, tw.data(), sizeof(float2) * nx, cudaMemcpyHostToDevice);
	twiddles(tw, ny);
	if (cudaMalloc(&d_twy_, sizeof(float2) * ny) != cudaSuccess) return 4;
	cudaMemcpy(d_twy_, tw.data(), sizeof(float2) * ny, cudaMemcpyHostToDevice);
	// phase-grating aperture (src/JEElaSca.cpp:586-609): 1/(nx ny) inside
	// 2/3 of the smaller Nyquist frequency, 0 outside; float arithmetic as there
	const int nx2 = (nx - nx % 2) >> 1, ny2 = (ny - ny % 2) >> 1;
	const float itogx = 1.f / a, itogy = 1.f / b;
	kmax_ = std::min((float)nx2 * itogx, (float)ny2 * itogy);
	const float kthr = kmax_ * 0.6666667f;
	const float ftrn = 1.f / (float)nx / (float)ny;
	std::vector<float2> ap((size_t)nx * ny);
	for (int j = 0; j < ny; j++) {
		const float qy = (float)(((j + ny2) % ny) - ny2) * itogy;
		for (int i = 0; i < nx; i++) {
			const float qx = (float)(((i + nx2) % nx) - nx2) * itogx;
			const float gm = std::sqrt(qx * qx + qy * qy);
			ap[(size_t)j * nx + i] = make_float2(gm > kthr ? 0.f : ftrn, 0.f);
		}
	}
	if (cudaMalloc(&d_ap2_, sizeof(float2) * ap.size()) != cudaSuccess) return 4;
	cudaMemcpy(d_ap2_, ap.data(), sizeof(float2) * ap.size(), cudaMemcpyHostToDevice);
	status_ |= 1;
	return 0;
}

int PgrGen::SetPhysics(float ekv, int thermal, int bwl_pot, int bwl_pgr)
{
	if (!(ekv > 0.f) || thermal < 0 || thermal > 2) return 1;
	ClearSites();
	fq_valid_ = false;
	ekv_ = ekv;
	thermal_ = thermal;
	bwl_pot_ = bwl_pot ? 1 : 0;
	bwl_pgr_ = bwl_pgr ? 1 : 0;
	// electron wavelength as CJEElaSca computes it (src/JEElaSca.cpp:826), float
	const float wlelkev = (float)(kC0 * kHPL / kQEL * 1.0E+6);
	const float eel0kev = (float)(kME0 * kC0 * kC0 / kQEL / 1000.);
	wl_ = wlelkev / std::sqrt(ekv * (ekv + 2.f * eel0kev));
	status_ |= 2;
	return 0;
}

int PgrGen::SetFormFactors(int ntype, int nk, float sk, const float* ff, const float* biso)
{
	if (ntype < 1 || nk < 2 || !(sk > 0.f) || ff == nullptr) return 1;
	ClearSites();
	fq_valid_ = false;
	dfree(d_ff_);
	d_ff_ = nullptr;
	if (cudaMalloc(&d_ff_, sizeof(float2) * (size_t)ntype * nk) != cudaSuccess) return 4;
	if (cudaMemcpy(d_ff_, ff, sizeof(float2) * (size_t)ntype * nk, cudaMemcpyHostToDevice) != cudaSuccess) return 5;
	ntype_ = ntype;
	nk_ = nk;
	sk_ = sk;
	biso_.assign(ntype, 0.f);
	if (biso) biso_.assign(biso, biso + ntype);
	status_ |= 4;
	return 0;
}

int PgrGen::BuildSites(int natom, const float* atoms, float cz, SiteSet** out)
{
	*out = nullptr;
	for (SiteSet& t : sets_) {
		if ((int)t.key.size() == 5 * natom + 1 && t.key[5 * natom] == cz &&
			std::memcmp(t.key.data(), atoms, sizeof(float) * 5 * natom) == 0) {
			t.used = ++use_clock_;
			*out = &t;
			nsite_ = t.nsite;
			natom_ = t.natom;
			return 0;
		}
	}
	// CStructure::SetAtomSites (src/Structure.cpp:441-491): an atom joins the
	// first site closer than 0.05 nm, else opens a new one; a site sits at the
	// occupancy-weighted mean of its atoms, with their occupancy-weighted Biso
	struct Site { double x, y, z, occ, bocc; std::vector<int> at; };
	std::vector<Site> sites;
	std::vector<int> site_of(natom);
	for (int i = 0; i < natom; i++) {
		const float* r = atoms + 5 * i;
		const int t = (int)r[4];
		if (t < 0 || t >= ntype_ || !(r[3] >= 0.f)) return 2;
		int fs = -1;
		for (size_t s = 0; s < sites.size(); s++) {
			const double dx = (r[0] - sites[s].x) * a_, dy = (r[1] - sites[s].y) * b_, dz = (r[2] - sites[s].z) * cz;
			if (std::sqrt(dx * dx + dy * dy + dz * dz) < kSiteClose) { fs = (int)s; break; }
		}
		if (fs < 0) {
			sites.push_back({r[0], r[1], r[2], r[3], (double)biso_[t] * r[3], {i}});
			site_of[i] = (int)sites.size() - 1;
			continue;
		}
		Site& S = sites[fs];
		S.at.push_back(i);
		double o = 0, px = 0, py = 0, pz = 0, bo = 0;
		for (int k : S.at) {
			const float* q = atoms + 5 * k;
			o += q[3]; px += q[0] * (double)q[3]; py += q[1] * (double)q[3]; pz += q[2] * (double)q[3];
			bo += (double)biso_[(int)q[4]] * q[3];
		}
		if (o > 0) { S.x = px / o; S.y = py / o; S.z = pz / o; }
		S.occ = o;
		S.bocc = bo;
		site_of[i] = fs;
	}
	const int nsite = (int)sites.size();
	std::vector<double2> base(nsite);
	std::vector<double> ux(nsite), uy(nsite);
	const double rsq8pi2 = 1.0 / std::sqrt(8.0 * kPi * kPi);
	for (int s = 0; s < nsite; s++) {
		base[s] = make_double2(sites[s].x, sites[s].y);
		const double bs = sites[s].occ > 0 ? sites[s].bocc / sites[s].occ : 0.0;
		const double u = (thermal_ == 2 && bs > 0) ? std::sqrt(bs) * rsq8pi2 : 0.0;   // nm
		ux[s] = u / a_;
		uy[s] = u / b_;
	}
	// atoms ordered by type for the synthesis kernel
	std::vector<int> order(natom);
	for (int i = 0; i < natom; i++) order[i] = i;
	std::stable_sort(order.begin(), order.end(), [&](int p, int q) { return (int)atoms[5 * p + 4] < (int)atoms[5 * q + 4]; });
	std::vector<int> asite(natom), tstart(ntype_ + 1, 0);
	std::vector<float> aocc(natom);
	for (int k = 0; k < natom; k++) {
		asite[k] = site_of[order[k]];
		aocc[k] = atoms[5 * order[k] + 3];
		tstart[(int)atoms[5 * order[k] + 4] + 1]++;
	}
	for (int t = 0; t < ntype_; t++) tstart[t + 1] += tstart[t];
	nsite_ = nsite;
	natom_ = natom;
	// a new set (the least recently used one of eight is replaced)
	constexpr size_t kMaxSets = 8;
	SiteSet* set = nullptr;
	if (sets_.size() < kMaxSets) {
		sets_.emplace_back();
		set = &sets_.back();
	}
	else {
		set = &sets_[0];
		for (SiteSet& t : sets_)
			if (t.used < set->used) set = &t;
		if (stream_) cudaStreamSynchronize(stream_);   // its buffers may still be read
		set->release();
	}
	cudaStream_t s = stream_;
	size_t c0 = 0, c1 = 0, c2 = 0, c3 = 0, c4 = 0, c5 = 0;
	int e;
	if ((e = dput(set->base, c0, base.data(), base.size(), s))) return e;
	if ((e = dput(set->ux, c1, ux.data(), ux.size(), s))) return e;
	if ((e = dput(set->uy, c2, uy.data(), uy.size(), s))) return e;
	if ((e = dput(set->asite, c3, asite.data(), asite.size(), s))) return e;
	if ((e = dput(set->aocc, c4, aocc.data(), aocc.size(), s))) return e;
	if ((e = dput(set->tstart, c5, tstart.data(), tstart.size(), s))) return e;
	set->key.assign(atoms, atoms + 5 * (size_t)natom);
	set->key.push_back(cz);
	set->nsite = nsite;
	set->natom = natom;
	set->used = ++use_clock_;
	*out = set;
	// the host vectors must outlive the asynchronous copies
	return cudaStreamSynchronize(s) == cudaSuccess ? 0 : 5;
}

int PgrGen::Calculate(int natom, const float* atoms, float cz, int ngr, unsigned long long seed, float2* d_dst,
	float* host_out)
{
	if ((status_ & 7) != 7) return 1;
	if (ngr < 1 || natom < 0 || (natom > 0 && atoms == nullptr) || !(cz > 0.f)) return 3;
	SiteSet* set = nullptr;
	int e = BuildSites(natom, atoms, cz, &set);
	if (e) return e;
	const long long N = (long long)nx_ * ny_;
	cudaStream_t s = stream_;
	if ((e = dput(d_buf_, cap_buf_, (const float2*)nullptr, (size_t)(ngr * N), s))) return e;
	float2* dst = d_dst;
	if (dst == nullptr) {
		if ((e = dput(d_out_, cap_out_, (const float2*)nullptr, (size_t)(ngr * N), s))) return e;
		dst = d_out_;
	}
	PgrArgs p;
	p.out = d_buf_;
	p.gstride = N;
	p.nx = nx_;
	p.ny = ny_;
	p.ngr = ngr;
	p.nsite = nsite_;
	p.atom_site = set->asite;
	p.atom_occ = set->aocc;
	p.type_start = set->tstart;
	p.ntype = ntype_;
	p.ff = d_ff_;
	p.nk = nk_;
	p.sk = sk_;
	p.itogx = 1.f / a_;
	p.itogy = 1.f / b_;
	p.kmax = kmax_;
	p.bwl_pot = bwl_pot_;
	// t = exp(i c V'), c = lambda cz / (4 pi vol), vol = a b cz (orthorhombic)
	p.cphase = (double)wl_ / (4.0 * kPi * (double)a_ * (double)b_);
	p.twx = d_twx_;
	p.twy = d_twy_;
	if (natom > 0) {
		if ((e = dput(d_pos_, cap_pos_, (const double2*)nullptr, (size_t)ngr * nsite_, s))) return e;
		if (launch_pgr_sites(d_pos_, set->base, set->ux, set->uy, nsite_, ngr, seed, s) != cudaSuccess) return 6;
		p.site_pos = d_pos_;
		if (!fq_valid_) {
			// the fq table lives as long as the setup: sized once per grid and type count
			dfree(d_fq_);
			d_fq_ = nullptr;
			if (cudaMalloc(&d_fq_, sizeof(float2) * (size_t)ntype_ * N) != cudaSuccess) return 4;
			if (launch_pgr_fq(p, d_fq_, s) != cudaSuccess) return 6;
			fq_valid_ = true;
		}
		p.fq = d_fq_;
		p.natom = natom_;
		// phase tables in groups of gratings of at most 64 MiB (L2-resident
		// while the synthesis reads each entry once per tile)
		const size_t per = (size_t)natom_ * (size_t)(nx_ + ny_);
		const int ng = (int)std::max<size_t>(1, std::min<size_t>((size_t)std::min(ngr, 65535),
			((size_t)64 << 20) / (sizeof(float2) * std::max<size_t>(per, 1))));
		if ((e = dput(d_tab_, cap_tab_, (const float2*)nullptr, per * ng, s))) return e;
		for (int g0 = 0; g0 < ngr; g0 += ng) {
			PgrArgs q = p;
			q.ngr = std::min(ng, ngr - g0);
			q.site_pos = d_pos_ + (size_t)g0 * nsite_;
			q.out = d_buf_ + (size_t)g0 * N;
			q.tx = d_tab_;
			q.ty = d_tab_ + (size_t)natom_ * nx_ * q.ngr;
			if (launch_pgr_phase(q, s) != cudaSuccess) return 6;
			if (launch_pgr_synth(q, s) != cudaSuccess) return 6;
		}
		if (launch_pgr_rows_inv(p, s) != cudaSuccess) return 6;
	}
	else if (cudaMemsetAsync(d_buf_, 0, sizeof(float2) * ngr * N, s) != cudaSuccess) {
		return 6;
	}
	if (bwl_pgr_) {
		if (launch_pgr_cols(p, d_buf_, d_buf_, kPgrColExpFt, s) != cudaSuccess) return 7;
		PassArgs r;
		r.work = d_buf_;
		r.wstride = N;
		r.nx = nx_;
		r.ny = ny_;
		r.nwave = ngr;
		r.twx = d_twx_;
		r.twy = d_twy_;
		r.mul = d_ap2_;
		const PlanOps* po = plan_get(nx_, 0);
		if (po == nullptr || po->row(r, s) != cudaSuccess) return 7;
		if (launch_pgr_cols(p, d_buf_, dst, kPgrColInv, s) != cudaSuccess) return 7;
	}
	else if (launch_pgr_cols(p, d_buf_, dst, kPgrColExp, s) != cudaSuccess) {
		return 7;
	}
	if (host_out) {
		if (cudaMemcpyAsync(host_out, dst, sizeof(float2) * ngr * N, cudaMemcpyDeviceToHost, s) != cudaSuccess) return 5;
		if (cudaStreamSynchronize(s) != cudaSuccess) return 5;
	}
	return 0;
}

} // namespace jms
