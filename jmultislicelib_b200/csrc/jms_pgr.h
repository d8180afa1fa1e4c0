// jms_pgr.h -- on-device phase-grating generation.
//
// Device counterpart of CJEElaSca::CalculatePhasegratingGPU / ..CPU
// (src/JEElaSca.cpp:812-1159) in its 2-D projection mode:
//
//   pot(q)  = sum_type ff2d_type(q) ap1(q) sum_atom occ exp(-2 pi i q.r)
//             with ff2d_type(q) = f_type(|q|) [ap1(q)], f linearly
//             interpolated from the radial table (CAtomType::GetFormFactor,
//             src/Atoms.cpp:414-436), ap1 the smooth potential band limit
//             (src/JEElaSca.cpp:597-600), applied twice as the reference does
//             (PrepareScatteringFunctions :738-739 and the add :934);
//   V'(r)   = IFT[pot] (unscaled, e^{+i});
//   t(r)    = exp(i c V'(r)),  c = lambda cz / (4 pi vol): the reference's
//             POT_SCA / vol and PGR_SIG cz lambda, whose constant product is
//             1 / (4 pi) (src/JEElaSca.cpp:947, 956-963, JEElaSca.h:88-94);
//   t       = IFT[ FT[t] ap2 ],  ap2 = 1/(nx ny) for |q| <= 2/3 kmax, else 0
//             (m_bwl_pgr, :965-969, aperture :602-609).
//
// Design: one synthesis kernel per batch of gratings (every grating a new
// draw of the site displacements in the quantum-excitation-of-phonons model,
// or the same sites), then the line plans of the multislice passes for the
// transforms: a row IFT, a column pass IFT_y -> exp(i c V') -> FT_y, the
// multislice row pass FT_x -> x ap2 -> IFT_x, and a column IFT_y that writes
// the gratings to their destination (the library's grating store).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace jms {

struct PgrArgs {
	float2* out = nullptr;          // [ngr][ny][nx]
	long long gstride = 0;          // elements between gratings
	int nx = 0, ny = 0, ngr = 0;
	// structure: sites with per-grating positions, atoms sorted by type
	const double2* site_pos = nullptr;  // [ngr][nsite] fractional (x/a, y/b)
	int nsite = 0;
	const int* atom_site = nullptr;     // [natom]
	const float* atom_occ = nullptr;    // [natom]
	const int* type_start = nullptr;    // [ntype + 1] atom ranges per type
	int ntype = 0;
	// radial form factors [ntype][nk] (complex, nm), sampling sk (1/nm/sample)
	const float2* ff = nullptr;
	int nk = 0;
	float sk = 0.f;
	float itogx = 0.f, itogy = 0.f;     // 1/a, 1/b as the reference's float helpers
	float kmax = 0.f;                   // min(nyq_x / a, nyq_y / b)
	int bwl_pot = 0;
	// precomputed tables of the synthesis: f_t(|q|) ap(q)^2 per type and pixel
	// [ntype][ny][nx]; translation phases per grating and atom (atoms in type
	// order), ex [ngr][natom][nx] and occ * ey [ngr][natom][ny]
	const float2* fq = nullptr;
	float2* tx = nullptr;
	float2* ty = nullptr;
	int natom = 0;
	// potential -> grating
	double cphase = 0.0;                // c of t = exp(i c V')
	const float2* twx = nullptr;
	const float2* twy = nullptr;
};

// QEP site displacement draws: pos[g][s] = base[s] + u[s] * (n1 / a, n2 / b),
// n1, n2 standard normal from a counter-based generator (splitmix64 of
// seed, g, s; Box-Muller).
cudaError_t launch_pgr_sites(double2* pos, const double2* base, const double* ux_frac, const double* uy_frac,
	int nsite, int ngr, unsigned long long seed, cudaStream_t s);
// fq[t][iy][ix] = f_t(|q|) (ap(q)^2 with bwl_pot) for the grid and form factors of p
cudaError_t launch_pgr_fq(const PgrArgs& p, float2* fq, cudaStream_t s);
// translation-phase tables p.tx, p.ty of the p.ngr gratings at p.site_pos
cudaError_t launch_pgr_phase(const PgrArgs& p, cudaStream_t s);
// potential spectra of p.ngr gratings from the tables p.fq, p.tx, p.ty
cudaError_t launch_pgr_synth(const PgrArgs& p, cudaStream_t s);

// transforms with the default plan of the length (nx for rows, ny for columns)
enum PgrColMode { kPgrColExpFt = 0, kPgrColExp = 1, kPgrColInv = 2 };
bool pgr_supported(int nx, int ny);
cudaError_t launch_pgr_rows_inv(const PgrArgs& p, cudaStream_t s);            // in place, IFT_x
cudaError_t launch_pgr_cols(const PgrArgs& p, const float2* src, float2* dst, int mode, cudaStream_t s);

} // namespace jms
