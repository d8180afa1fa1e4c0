/*
 * ref_driver.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * A thin extern "C" driver over the reference's own CJMultiSlice class
 * (src/JMultiSlice.h:185-738), compiled together with the reference sources
 * by oracle/Makefile into oracle/_ref/libjms_ref.so.  Tests use it to make
 * golden vectors and to check the FP64 oracle; bench.py's reference arm uses
 * it to time the reference CPU path (CPUMultislice on MKL DFTI).  Nothing in
 * the product links or loads this file.
 *
 * Every function forwards to the reference method of the same name; no
 * reference source is copied here.  ref_pgr drives the reference's phase
 * grating calculation (CJEElaSca, src/JEElaSca.h:98-273) on its CPU path.
 */
#include "JMultiSlice.h"
#include "JEElaSca.h"
#include "prm_slice_file_info.h"
#include <algorithm>
#include <atomic>
#include <chrono>
#include <dlfcn.h>
#include <thread>
#include <fstream>
#include <vector>
#include <string>
#include <cstring>

// Exposes protected reference methods needed for golden vectors.
class RefJMS : public CJMultiSlice {
public:
	using CJMultiSlice::GetRandomVariantSequence; // JMultiSlice.cpp:1571
	fcmplx* cpu_wave(int ithread) { // thread wave slot after OffsetIncomingWave (JMultiSlice.cpp:2024)
		return m_h_wav + (int64_t)m_nscx * m_nscy * ithread;
	}
};

// Exposes the prepared atom types (radial form factors) of CJEElaSca.
class RefEElaSca : public CJEElaSca {
public:
	const std::vector<CAtomType>& types() const { return m_vTypes; }
};

extern "C" {

void* ref_create(void) { return new RefJMS(); }
void ref_destroy(void* h) { delete (RefJMS*)h; }

float ref_set_high_tension(void* h, float ht) { ((RefJMS*)h)->SetHighTension(ht); return ((RefJMS*)h)->GetWaveLength(); }
void ref_set_grid(void* h, int nx, int ny, float a, float b, float c)
{
	((RefJMS*)h)->SetGridSize(nx, ny);
	((RefJMS*)h)->SetSupercellSize(a, b, c);
}
void ref_seed(void* h, int seed) { ((RefJMS*)h)->SeedRngEx(seed); }

int ref_phase_grating_setup(void* h, int code, int nx, int ny, int nslc, int nvarmax, int* nslcvar)
{ return ((RefJMS*)h)->PhaseGratingSetup(code, nx, ny, nslc, nvarmax, nslcvar); }
int ref_object_slice_setup(void* h, int nobjslc, int* objslc)
{ return ((RefJMS*)h)->ObjectSliceSetup(nobjslc, objslc); }
int ref_propagator_setup(void* h, int code, int npro, int* proidx)
{ return ((RefJMS*)h)->PropagatorSetup(code, npro, proidx); }
int ref_detector_setup(void* h, int code, int ndetper, int ndetint, int imagedet, int nthreads)
{ return ((RefJMS*)h)->DetectorSetup(code, ndetper, ndetint, imagedet, nthreads); }
int ref_set_phase_grating(void* h, int code, int islc, int nvar, float* pgr)
{ return ((RefJMS*)h)->SetPhaseGratingData(code, islc, nvar, (fcmplx*)pgr); }
int ref_set_propagator(void* h, int code, int ipro, float* pro)
{ return ((RefJMS*)h)->SetPropagatorData(code, ipro, (fcmplx*)pro); }
int ref_set_detector(void* h, int code, int idet, float* det, int msklen, int* msk)
{ return ((RefJMS*)h)->SetDetectorData(code, idet, det, msklen, msk); }
int ref_init_core(void* h, int code, int nthreads) { return ((RefJMS*)h)->InitCore(code, nthreads); }
int ref_set_incident_wave(void* h, int code, float* wav) { return ((RefJMS*)h)->SetIncidentWave(code, (fcmplx*)wav); }
int ref_set_phaseplate(void* h, int code, float* ppl) { return ((RefJMS*)h)->SetIncidentWavePhaseplate(code, ppl); }
int ref_offset_incoming_wave(void* h, int code, float dx, float dy, float dz, int ithread, int ibtx, int ibty)
{ return ((RefJMS*)h)->OffsetIncomingWave(code, dx, dy, dz, ithread, ibtx, ibty); }
int ref_cpu_multislice(void* h, int islc0, int accmode, float weight, int ithread)
{ return ((RefJMS*)h)->CPUMultislice(islc0, accmode, weight, ithread); }
int ref_gpu_multislice(void* h, int islc0, int accmode, float weight)
{ return ((RefJMS*)h)->GPUMultislice(islc0, accmode, weight); }
int ref_get_result(void* h, int code, int which, float* dst, int ithread)
{ return ((RefJMS*)h)->GetResult(code, which, dst, ithread); }
int ref_get_avg_result(void* h, int code, int which, float* dst, float* wgt, int ithread)
{ float w = 0.f; int e = ((RefJMS*)h)->GetAvgResult(code, which, dst, w, ithread); *wgt = w; return e; }
int ref_num_det_planes(void* h) { return ((RefJMS*)h)->GetDetetionSliceNum(); }
int ref_unscramble_hash(void* h, unsigned int* hash) { return ((RefJMS*)h)->GetUnscrambleHash(hash); }
int ref_variant_sequence(void* h, int* out) { return ((RefJMS*)h)->GetRandomVariantSequence(out); }
void ref_cpu_wave(void* h, int ithread, float* dst, int n)
{ memcpy(dst, ((RefJMS*)h)->cpu_wave(ithread), sizeof(fcmplx) * (size_t)n); }
int ref_detection_planes(void* h, int ndetper, int nobjslc, int* det_objslc)
{ return ((RefJMS*)h)->SetDetectionPlanes(ndetper, nobjslc, det_objslc); }
int ref_cleanup(void* h) { return ((RefJMS*)h)->Cleanup(); }

// CalculateProbeWaveFourier (JMultiSlice.cpp:983) with the public CJProbeParams
// fields (JProbeGen.h:60-94); abrr holds 2*24 coefficients [nm].
int ref_calc_probe(void* h, float alpha, float alpha_rs, float alpha_x0, float alpha_y0,
	float alpha_asym, float alpha_adir, float btx, float bty, const float* abrr, int nabrr2, float* wav)
{
	CJProbeParams prm;
	prm.m_alpha = alpha; prm.m_alpha_rs = alpha_rs;
	prm.m_alpha_x0 = alpha_x0; prm.m_alpha_y0 = alpha_y0;
	prm.m_alpha_asym = alpha_asym; prm.m_alpha_adir = alpha_adir;
	prm.m_btx = btx; prm.m_bty = bty;
	int nac = 2 * prm.GetAberrationNum();
	for (int i = 0; i < nac && i < nabrr2; i++) prm.m_abrr_coeff[i] = abrr[i];
	return ((RefJMS*)h)->CalculateProbeWaveFourier(&prm, (fcmplx*)wav);
}
int ref_calc_propagator(void* h, float fthick, float otx, float oty, int ntype, float* pro)
{ return ((RefJMS*)h)->CalculatePropagator(fthick, otx, oty, (fcmplx*)pro, ntype); }
int ref_calc_ring_detector(void* h, float beta0, float beta1, float phi0, float phi1,
	float th0x, float th0y, const char* profile, float* det, int* msklen, int* msk, int kmom1)
{
	int ml = 0;
	int e = ((RefJMS*)h)->CalculateRingDetector(beta0, beta1, phi0, phi1, th0x, th0y,
		std::string(profile ? profile : ""), det, ml, msk, kmom1);
	*msklen = ml;
	return e;
}

// Multi-threaded reference CPU scan, following the hybrid queue of the
// reference benchmark (test/JMSBench1/multislice.cpp:1236-1416): worker
// threads pull probe positions from a shared counter; per position they run
// nrepeat frozen-phonon passes of OffsetIncomingWave + CPUMultislice with
// weight 1/nrepeat and read the integrated detectors.  Each worker owns one
// CJMultiSlice object (the CPU path borrows the caller's host arrays, so the
// objects share gratings, propagators and detectors) and runs MKL
// sequentially, as the reference links mkl_sequential.
// objs: nthreads handles, each fully set up for CPU code with 1 thread channel.
// pos: npos (dx,dy) pairs [nm]; out: npos * ndetslc * ndet floats.
int ref_cpu_scan(void** objs, int nthreads, int npos, const float* pos, int nrepeat,
	int ndetout, float* out)
{
	std::atomic<int> next(0);
	std::atomic<int> err(0);
	std::vector<std::thread> pool;
	for (int t = 0; t < nthreads; t++) {
		pool.emplace_back([&, t]() {
			// MKL runs sequentially in this worker: its OpenMP layer reads the
			// thread count of the calling thread, which is set to 1 here
			typedef void (*omp_set_t)(int);
			if (omp_set_t f = (omp_set_t)dlsym(RTLD_DEFAULT, "omp_set_num_threads")) f(1);
			RefJMS* jms = (RefJMS*)objs[t];
			float w = 1.f / (float)nrepeat;
			for (;;) {
				int ip = next.fetch_add(1);
				if (ip >= npos) break;
				for (int ir = 0; ir < nrepeat; ir++) {
					int e = jms->OffsetIncomingWave(_JMS_CODE_CPU, pos[2 * ip], pos[2 * ip + 1], 0.f, 0);
					if (e == 0) e = jms->CPUMultislice(0, ir > 0 ? 1 : 0, w, 0);
					if (e != 0) { err.store(e); return; }
				}
				jms->GetResult(_JMS_CODE_CPU, _JMS_DETECT_INTEGRATED, out + (size_t)ip * ndetout, 0);
			}
		});
	}
	for (auto& th : pool) th.join();
	return err.load();
}

// The reference GPU path (CJMultiSlice::GPUMultislice on cuFFT and the
// ArrayOps kernels, src/JMultiSlice.cpp:4513-4677) driven per probe position
// as the reference benchmark drives it (test/JMSBench1/multislice.cpp:551-620):
// nrepeat frozen-phonon passes of OffsetIncomingWave + GPUMultislice (weight
// 1/nrepeat, accumulating after the first), then GetResult of the integrated
// detectors.  h: one object set up for GPU code.  *seconds: wall time of the
// loop; every reference GPU call ends with a device synchronisation, so it is
// the device time of the work.  out: npos * ndetout floats.
int ref_gpu_scan(void* h, int npos, const float* pos, int nrepeat, int ndetout, float* out, double* seconds)
{
	RefJMS* jms = (RefJMS*)h;
	const float w = 1.f / (float)nrepeat;
	auto t0 = std::chrono::steady_clock::now();
	for (int ip = 0; ip < npos; ip++) {
		for (int ir = 0; ir < nrepeat; ir++) {
			int e = jms->OffsetIncomingWave(_JMS_CODE_GPU, pos[2 * ip], pos[2 * ip + 1], 0.f, 0);
			if (e == 0) e = jms->GPUMultislice(0, ir > 0 ? 1 : 0, w);
			if (e != 0) return e;
		}
		int e = jms->GetResult(_JMS_CODE_GPU, _JMS_DETECT_INTEGRATED, out + (size_t)ip * ndetout, 0);
		if (e != 0) return e;
	}
	auto t1 = std::chrono::steady_clock::now();
	if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
	return 0;
}

void ref_set_slice_thickness(void* h, int islc, float t) { ((RefJMS*)h)->SetSliceThickness(islc, t); }
void ref_set_plasmon(void* h, int use, float q_e, float q_c, float mfp, unsigned int nexmax)
{
	((RefJMS*)h)->SetPlasmonMC(use != 0, q_e, q_c, mfp, nexmax);
}

// EMS slice-file header through the bench driver's prm_slice_file_info
// (test/JMSBench1/prm_slice_file_info.cpp): load_ems_header of a file, and a
// file whose header comes from save_ems_header (data appended at 8192).
// ints: nx, ny, nvar, content, version; offs: data, table; f: thickness, ekv, sx, sy.
int ref_sli_read_header(const char* path, int* ints, unsigned long long* offs, float* f, char* title)
{
	prm_slice_file_info h;
	std::ifstream fs(path, std::ios::binary);
	if (!fs.is_open()) return 2;
	int e = h.load_ems_header(&fs);
	if (e) return e;
	ints[0] = (int)h.grid_x; ints[1] = (int)h.grid_y; ints[2] = (int)h.num_var; ints[3] = (int)h.data_type;
	ints[4] = (int)h.ver;
	offs[0] = h.data_offset; offs[1] = h.structure_offset;
	f[0] = h.sz; f[1] = h.ekv; f[2] = h.sx; f[3] = h.sy;
	std::memcpy(title, h.s_slc_name, 40);
	return 0;
}

int ref_sli_write(const char* path, int nx, int ny, int nvar, int content, float thickness, float ekv, float sx,
	float sy, const char* title, const float* pgr)
{
	prm_slice_file_info h;
	h.grid_x = (unsigned)nx; h.grid_y = (unsigned)ny; h.num_var = (unsigned)nvar; h.data_type = (unsigned)content;
	h.data_offset = 8192; h.structure_offset = 0x1100;
	h.sz = thickness; h.ekv = ekv; h.sx = sx; h.sy = sy;
	std::memset(h.s_slc_name, 0, 40);
	std::strncpy(h.s_slc_name, title, 40);
	std::ofstream fs(path, std::ios::binary);
	if (!fs.is_open()) return 2;
	int e = h.save_ems_header(&fs);
	if (e) return e;
	std::vector<char> pad(8192 - 0x1100, 0);
	fs.write(pad.data(), pad.size());
	fs.write((const char*)pgr, sizeof(float) * 2 * (size_t)nx * ny * nvar);
	return fs.good() ? 0 : 6;
}

// CJMultiSlice::ReadoutDetAvg (src/JMultiSlice.cpp:2667-2945).
int ref_readout_det_avg(void* h, int whichcode, int whichresult, float* dst, float* weight, int ithread)
{
	float w = 0.f;
	int e = ((RefJMS*)h)->ReadoutDetAvg(whichcode, whichresult, dst, w, ithread);
	if (weight) *weight = w;
	return e;
}

// Phase grating(s) of one structure slice by the reference's CJEElaSca on the
// CPU path: CStructure::AddAtom per atom (Z, Biso [nm^2], occupancy,
// fractional x, y, z), SetAtomSites(0.05), cell (a, b, c) [nm] at 90 degrees
// with the identity basis; SetGrid(nx, ny, 1, 0), SetPhysics(ekv, 0, absorb,
// abf, thermal), CalculateFormFactors, PrepareScatteringFunctions(-1, 1),
// then nrep x CalculatePhasegratingCPU (thread 0) after SeedRngEx(seed).
// Outputs: pgr [nrep][ny][nx] complex, atom_type [natom] (type index of each
// atom), ff [ntype][nk] complex and sk of the prepared types (ff may be NULL;
// *nk_io in: capacity per type, out: nk), *ntype_out, *seconds (time of the
// nrep grating calls).  Returns 0 or the first reference error + 100 * stage.
int ref_pgr(int nx, int ny, float a, float b, float c, float ekv, int thermal, int absorb, float abf, int natom,
	const int* Z, const float* biso, const float* occ, const float* pos, int nrep, int seed, float* pgr,
	int* atom_type, float* ff, int* nk_io, float* sk_out, int* ntype_out, double* seconds)
{
	CStructure st;
	st.m_vCellSize = CV3D(a, b, c);
	st.m_vCellAngles = CV3D(90.f, 90.f, 90.f);
	for (int i = 0; i < natom; i++)
		st.AddAtom(Z[i], 0.f, biso[i], occ[i], pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
	st.SetAtomSites(0.05f);
	RefEElaSca E;
	int e;
	if ((e = E.SetStructure(st))) return 100 + e;
	if ((e = E.SetGrid((unsigned)nx, (unsigned)ny, 1u, 0u))) return 200 + e;
	if ((e = E.SetPhysics(ekv, 0u, (unsigned)absorb, abf, (unsigned)thermal))) return 300 + e;
	if ((e = E.CalculateFormFactors(false))) return 400 + e;
	if ((e = E.PrepareScatteringFunctions(-1, 1, false))) return 500 + e;
	E.SeedRngEx(seed);
	const size_t N = (size_t)nx * ny;
	auto t0 = std::chrono::steady_clock::now();
	for (int r = 0; r < nrep; r++) {
		if ((e = E.CalculatePhasegratingCPU(&st, (fcmplx*)(pgr + 2 * N * r), 0))) return 600 + e;
	}
	auto t1 = std::chrono::steady_clock::now();
	if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
	for (int i = 0; i < natom; i++) atom_type[i] = st.m_vAtoms[i].m_nAtomTypeIndex;
	// the prepared radial tables: CAtomType::CopyFormFactors (src/Atoms.cpp:106-127)
	// never hands its buffer back, so the samples are read with GetFormFactor
	// at q = k sk (linear interpolation there returns the sample); nk and sk
	// as CalculateFormFactors sets them (src/JEElaSca.cpp:459-462)
	const auto& ty = E.types();
	if (ntype_out) *ntype_out = (int)ty.size();
	const int nk = 12 * std::max(std::max(nx, ny), 1);
	const float sk = std::max(std::max((float)nx / a, (float)ny / b), 1.f / c) / (float)nk;
	if (nk_io) {
		const int cap = *nk_io;
		*nk_io = nk;
		if (ff && nk <= cap) {
			for (size_t t = 0; t < ty.size(); t++) {
				CAtomType& T = const_cast<CAtomType&>(ty[t]);
				for (int k = 0; k < nk; k++) {
					const fcmplx v = T.GetFormFactor(sk * (float)std::min(k, nk - 2), 1);
					ff[2 * ((size_t)cap * t + k)] = v.real();
					ff[2 * ((size_t)cap * t + k) + 1] = v.imag();
				}
			}
		}
	}
	if (sk_out) *sk_out = sk;
	return 0;
}

} // extern "C"
