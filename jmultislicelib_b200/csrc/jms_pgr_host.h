// jms_pgr_host.h -- on-device phase-grating generator (host object), the
// counterpart of CJEElaSca (src/JEElaSca.h:98-273) in its 2-D projection mode.
#pragma once
#include <cuda_runtime.h>
#include <vector>

namespace jms {

class PgrGen {
public:
	PgrGen() = default;
	~PgrGen();
	PgrGen(const PgrGen&) = delete;
	PgrGen& operator=(const PgrGen&) = delete;

	// grid nx x ny over the orthorhombic cell a x b [nm] (CJEElaSca::SetGrid
	// and the structure's cell); 8 = unsupported grid size
	int SetGrid(int nx, int ny, float a, float b);
	// beam energy [keV]; thermal model 0 none, 1 Debye-Waller factors (part of
	// the form-factor tables), 2 QEP site displacements; band limits of the
	// potential (m_bwl_pot) and of the grating (m_bwl_pgr)
	int SetPhysics(float ekv, int thermal, int bwl_pot, int bwl_pgr);
	// radial form factors ff [ntype][nk] complex (nm) sampled every sk 1/nm,
	// and the Biso [nm^2] of each type (QEP displacement amplitudes)
	int SetFormFactors(int ntype, int nk, float sk, const float* ff, const float* biso);
	// ngr gratings of one structure slice: atoms [natom][5] = fractional x, y,
	// z, occupancy, type; cz = slice thickness [nm].  Written to d_dst
	// ([ngr][ny][nx] on the device) or to an internal buffer, and copied to
	// host_out when given.  Errors: 1 incomplete setup, 2 bad atom type or
	// occupancy, 3 bad arguments, 4 allocation, 5 copy, 6 potential kernels,
	// 7 grating kernels.
	int Calculate(int natom, const float* atoms, float cz, int ngr, unsigned long long seed, float2* d_dst,
		float* host_out);
	void SetStream(cudaStream_t s) { stream_ = s; }
	void Reset();
	int nx() const { return nx_; }
	int ny() const { return ny_; }
	int nsite() const { return nsite_; }

private:
	// a structure slice prepared on the device: linked sites, atoms ordered by
	// type; kept for reuse while the setup is unchanged (the QEP form of a scan
	// regenerates the same slices every pass)
	struct SiteSet {
		std::vector<float> key;         // atoms (5 floats each), then cz
		int nsite = 0, natom = 0;
		double2* base = nullptr;
		double *ux = nullptr, *uy = nullptr;
		int *asite = nullptr, *tstart = nullptr;
		float* aocc = nullptr;
		unsigned long long used = 0;
		void release();
	};
	int BuildSites(int natom, const float* atoms, float cz, SiteSet** out);
	void ClearSites();
	std::vector<SiteSet> sets_;
	unsigned long long use_clock_ = 0;

	int status_ = 0;
	int nx_ = 0, ny_ = 0;
	float a_ = 0.f, b_ = 0.f, kmax_ = 0.f;
	float ekv_ = 0.f, wl_ = 0.f;
	int thermal_ = 0, bwl_pot_ = 0, bwl_pgr_ = 1;
	int ntype_ = 0, nk_ = 0;
	float sk_ = 0.f;
	std::vector<float> biso_;
	int nsite_ = 0, natom_ = 0;
	cudaStream_t stream_ = nullptr;
	float2* d_ff_ = nullptr;
	float2 *d_twx_ = nullptr, *d_twy_ = nullptr, *d_ap2_ = nullptr, *d_buf_ = nullptr, *d_out_ = nullptr;
	double2* d_pos_ = nullptr;
	size_t cap_buf_ = 0, cap_out_ = 0, cap_pos_ = 0;
	// synthesis tables: f_t(|q|) per type and pixel (valid while grid, physics
	// and form factors are unchanged), translation phases per grating group
	float2* d_fq_ = nullptr;
	bool fq_valid_ = false;
	float2* d_tab_ = nullptr;
	size_t cap_tab_ = 0;
};

} // namespace jms
