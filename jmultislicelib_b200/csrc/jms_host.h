// jms_host.h -- host side of the B200 multislice library.
//
// JmsB200 mirrors the GPU code path of the reference class CJMultiSlice
// (src/JMultiSlice.h:185-738): the same setup chain and status bits, the same
// generators, error codes and result layouts, with every computation on the
// device done by the fused sm_100a passes of jms_kernels.cu.  The reference's
// CPU code path (whichcode _JMS_CODE_CPU, CPUMultislice) is not part of this
// library: calls that ask for it return error code 1.
//
// Beyond the reference interface it adds a batched scan entry point that runs
// many probe positions and frozen-phonon passes through one stream.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <random>

#include "../../include/rng.h"
#include <string>
#include <vector>

namespace jms {

struct PlanOps;

// flags (numeric values of src/JMultiSlice.h:126-149)
enum : int {
	CODE_CPU = 1, CODE_GPU = 2,
	STATUS_PGR = 1, STATUS_OBJ = 2, STATUS_PRO = 4, STATUS_DET = 8, STATUS_CORE = 16,
	THRESHOLD_CORE = 15, THRESHOLD_CALC = 31,
	DET_INTEGRATED = 1, DET_IMAGE = 2, DET_DIFFRACTION = 4, DET_WAVEREAL = 8, DET_WAVEFOURIER = 16,
	DET_IMAGE_AVG = 32, DET_DIFFR_AVG = 64, DET_WAVER_AVG = 128, DET_WAVEF_AVG = 256,
};

// electron wavelength [nm] at the kinetic energy ht [keV] (src/JMultiSlice.cpp:372-378)
float wavelength_nm(float ht);

// public probe parameters of CJProbeParams (src/JProbeGen.h:60-94)
struct ProbeParams {
	float wl = 0.001969f;       // wavelength [nm] (overwritten from the high tension)
	float alpha = 0.025f;       // convergence semi-angle [mrad]
	float alpha_rs = 0.03f;     // relative aperture edge smoothness
	float alpha_x0 = 0.f, alpha_y0 = 0.f; // aperture centre [mrad]
	float alpha_asym = 0.f;     // relative aperture asymmetry
	float alpha_adir = 0.f;     // asymmetry direction [deg]
	float btx = 0.f, bty = 0.f; // beam tilt [mrad]
	float abrr[48] = {0};       // 24 aberrations (x, y) [nm], order of CJProbeGen's table
};

class JmsB200 {
public:
	JmsB200();
	~JmsB200();
	JmsB200(const JmsB200&) = delete;
	JmsB200& operator=(const JmsB200&) = delete;

	// ---- physics and grid (src/JMultiSlice.cpp:372-445)
	float SetHighTension(float ht);
	float GetHighTension() const { return ht_; }
	float GetWaveLength() const { return wl_; }
	void SetSupercellSize(float a, float b, float c) { a0_[0] = a; a0_[1] = b; a0_[2] = c; }
	void GetSupercellSize(float* a0) const { a0[0] = a0_[0]; a0[1] = a0_[1]; a0[2] = a0_[2]; }
	void SetGridSize(int nx, int ny) { nx_ = nx; ny_ = ny; }
	void GetGridSize(int& nx, int& ny) const { nx = nx_; ny = ny_; }
	void SetSliceThickness(int islc, float t);
	float GetSliceThickness(int islc) const;
	int GetDetetionSliceNum() const { return ndetslc_; }
	int GetObjectSliceNum() const { return nobjslc_; }
	int GetDetNum() const { return ndet_; }
	int SetDetectionPlanes(int ndetper, int nobjslc, int* det_objslc) const;
	int SetDetectionPlanesList(const int* slc_det, int nlist, int nobjslc, int* det_objslc) const;

	// ---- diffraction descan (src/JMultiSlice.cpp:1108-1162) and plasmon switch
	void DiffractionDescan(bool on) { descan_on_ = on ? 1 : 0; }
	void SetDiffractionDescanN(int whichcode, int ndx, int ndy);
	void SetDiffractionDescan(int whichcode, float dkx, float dky);
	void SetDiffractionDescanMRad(int whichcode, float dmx, float dmy);
	// bulk plasmon Monte-Carlo (src/JMultiSlice.cpp:973-981, src/JPlasmonMC.cpp)
	void SetPlasmonMC(bool use, float q_e, float q_c, float mfp, unsigned int nexmax);

	// ---- generators (host, as in the reference)
	int CalculateProbeWaveFourier(const ProbeParams& prm, float* wav) const;
	int CalculatePropagator(float fthick, float otx, float oty, float* pro, int ntype);
	int CalculateRingDetector(float beta0, float beta1, float phi0, float phi1, float theta0x, float theta0y,
		const char* sdsprofile, float* det, int* msklen, int* msk, int kmom1) const;

	// ---- setup chain (src/JMultiSlice.h:77-97)
	int PhaseGratingSetup(int whichcode, int nx, int ny, int nslc, int nvarmax, const int* nslcvar);
	int ObjectSliceSetup(int nobjslc, const int* objslc);
	int PropagatorSetup(int whichcode, int npro, const int* proidx);
	int DetectorSetup(int whichcode, int ndetper, int ndetint, int imagedet, int nthreads_CPU);
	int DetectorSetupList(int whichcode, const int* slc_det, int nlist, int ndetint, int imagedet, int nthreads_CPU);
	int SetPhaseGratingData(int whichcode, int islc, int nvar, const float* pgr);
	int SetPropagatorData(int whichcode, int ipro, const float* pro);
	int SetDetectorData(int whichcode, int idet, const float* det, int msklen, const int* msk);
	int InitCore(int whichcode, int nCPUthreads);
	int SetIncidentWave(int whichcode, const float* wav, bool bTranspose);
	int SetIncidentWavePhaseplate(int whichcode, const float* ppl, bool bTranspose);
	int ZeroIncidentWavePhaseplate(int whichcode);
	int GetUnscrambleHash(unsigned int* phash) const;
	int SetGPUPgrLoading(int npgrload);

	// ---- RNG (src/rng.cpp:30-74 semantics): the context's own generator, or
	// a caller's (CJMultiSlice::SetRng, src/JMultiSlice.cpp:347-370)
	void SeedRngEx(int nseed);
	void SetRng(CRng* prng) { rng_ = prng ? prng : &own_rng_; }
	CRng* GetRng() { return rng_; }
	int GetRandomVariantSequence(int* out);

	// ---- calculation
	int OffsetIncomingWave(int whichcode, float dx, float dy, float dz, int iThread, int ibtx, int ibty, bool bcppl);
	int SetIncomingWaveGPU(const float* wav, bool bTranspose);
	int GPUMultislice(int islc0, int accmode, float weight);
	int GetResult(int whichcode, int whichresult, float* dst, int iThread);
	int GetAvgResult(int whichcode, int whichresult, float* dst, float* weight, int iThread);
	// CJMultiSlice::ReadoutDetAvg (src/JMultiSlice.cpp:2667-2945), GPU branch:
	// detector readouts of the averaged waves
	int ReadoutDetAvg(int whichcode, int whichresult, float* dst, float* weight, int iThread);
	float GetImageAveragingWeight(int whichcode, int iThread) const;
	float GetWaveAveragingWeight(int whichcode, int iThread) const;
	int ResetImageAveraging(int whichcode, int iThread);
	int ResetWaveAveraging(int whichcode, int iThread);
	int ClearDetMem_d();
	int Cleanup();

	// ---- device / stream
	int SetStream(cudaStream_t s);
	cudaStream_t Stream() const { return stream_; }
	int SetCurrentGPU(int idev);
	int GetCurrentGPU() const;

	// ---- batched scan (addition): positions x frozen-phonon passes
	// Host-buffer form: pos [npos][2] (dx, dy) nm; out_int [npos][ndetslc][ndet];
	// out_bin [npos][ny/bin][nx/bin] (or null).  varseq [npass][nobjslc] or null
	// (then one GetRandomVariantSequence draw per pass).  Each pass weighs 1/npass.
	int ScanGPU(int npos, const float* pos, float dz, int npass, const int* varseq, float* out_int, float* out_bin,
		int bin);
	// Device-buffer form of the same (pointers on the device; asynchronous on
	// the library stream).  out_int is double [npos][ndetslc][ndet].
	int ScanGPUDevice(int npos, const float* d_pos, float dz, int npass, const int* varseq, double* d_out_int,
		float* d_out_bin, int bin);
	// Integrated detectors of caller-provided Fourier-space waves (device
	// pointers) with the current detector setup, allocating nothing
	// (jms_noalloc.cu); d_out is double [nwave][ndet], overwritten.
	int ReadoutDetectorsNoAlloc(const float* d_wav, int nwave, double* d_out, cudaStream_t s);
	int SetScanBatch(int nwave) { scan_batch_ = nwave > 0 ? nwave : scan_batch_; return 0; }
	// With a variant sequence and fewer positions than the scan batch, the scan
	// puts several frozen-phonon configurations of the positions into one
	// launch (on by default); off = one launch sequence per configuration.
	int SetPassFusion(int on) { fuse_passes_ = on ? 1 : 0; return 0; }
	// Line-plan choice (jms_sizes.h): Autotune times every candidate plan of
	// nx (row passes) and ny (column passes) on nwave waves of the current
	// setup and keeps the fastest; the choice is remembered per length for
	// later setups in this process.  SelectPlans sets them by index.
	int Autotune(int nwave, int reps, float* ms_row, float* ms_col, int* irow, int* icol);
	int SelectPlans(int irow, int icol);
	const char* PlanName(int axis) const;
	int GetScanBatch() const { return scan_batch_; }
	// device address of grating variants ivar .. ivar + nvar - 1 of structure
	// slice islc (nullptr if out of the setup), with the grating grid size
	float2* GratingSlot(int islc, int ivar, int nvar, int* npgx, int* npgy);
	long long KernelLaunches() const { return launches_; }
	// Per-pass device timing: with it on, every column / row pass launch is
	// bracketed by CUDA events on the library stream; PassTiming sums them.
	void SetPassTiming(int on);
	int PassTiming(double* ms_col, long long* n_col, double* ms_row, long long* n_row);
	int LastCudaError() const { return (int)last_cuda_; }
	// Arithmetic of the line transforms: 0 = FP32 passes (default), 1 = tensor-
	// core passes with BF16 hi+lo operands, 2 = tensor-core passes with FP16
	// hi+lo operands (jms_tc.cu).  The tensor-core passes run the steps without
	// readout for line lengths 256, 512, 1024 and 2048; readout steps, sub-frame
	// gratings, plasmon shifts and other lengths keep the FP32 passes.
	int SetPrecision(int mode);
	int GetPrecision() const { return prec_; }
	// 0, or 1 if a tensor-core pass reported an MMA wait that ran out (the
	// flag is cleared by the call); synchronises the library stream
	int TcStatus();
	long long TcLaunches() const { return tc_launches_; }
	// device scratch of at least n doubles, owned by the context (grown on
	// demand, freed with it); nullptr if the allocation fails
	double* Scratch(size_t n);
	// Control-variate scratch of the multi-fidelity scan on this (coarse)
	// context: successive calls get the two halves of a 4 n buffer in turn, so
	// a call may clear its half while the previous call's combine still reads
	// the other one.  *done is the event to record after the combine that
	// reads the half handed out; the call waits for its earlier record (a
	// never-recorded event is complete) before clearing the half.
	double* CvScratch(size_t n, cudaEvent_t* done);
	int Status() const { return status_gpu_; }

private:
	int gpu_ready(int need) const { return (status_gpu_ & need) == need; }
	int post(cudaError_t e, const char* where);
	int ensure_work(int nwave);
	int ensure_partial(int nwave);
	// d_mulw (with var == nullptr): per-slice per-wave grating offsets
	// [nobjslc][nwave] of waves from several phonon configurations; wave_pos > 0:
	// wave b is position b % wave_pos for the detector sums and binned patterns
	int run_slices(int nwave, int islc0, const int* var, float weight, const float2* entry_src, const double* d_shift,
		int ibtx, int ibty, const float* d_cppl, double* d_detint, float* d_bin, int bin, int nbx, int nby,
		const int* plas = nullptr, const int* d_plas_w = nullptr, const int* d_mulw = nullptr, int wave_pos = 0);
	// one slice of the plasmon Monte-Carlo (CJPlasmonMC::ScatGridMC); returns
	// the number of new excitations, (di, dj) the change of the pixel shift
	int plasmon_step(float dt, int* di, int* dj);
	void free_all();

	// parameters
	float ht_ = 0.f, wl_ = 0.f;
	float a0_[3] = {0.f, 0.f, 0.f};
	int nx_ = 0, ny_ = 0, npgx_ = 0, npgy_ = 0;
	int nscslc_ = 0, nslcvar_ = 0, nobjslc_ = 0, npro_ = 0, nprotype_ = 0;
	int ndet_ = 0, ndetper_ = 0, imagedet_ = 0, ndetslc_ = 0;
	int status_gpu_ = 0;
	std::vector<int> nvarslc_, objslc_, det_objslc_, proidx_, detmask_len_, fnx_, fny_;
	std::vector<long long> slcoffset_;
	// per propagator: Fourier rows (ky, scrambled index) in (k1, k2) are zero
	// everywhere (band limit); k1 = ny - 1 when every row has a nonzero value
	std::vector<int> pro_k1_, pro_k2_;
	int wav0_k1_ = 1 << 30, wav0_k2_ = 1 << 30;   // band of the incident wave's nonzero rows
	std::vector<float> slcthick_;
	// random numbers of the variant draws and plasmon paths
	CRng own_rng_;
	CRng* rng_ = &own_rng_;
	double unirand(double a, double b) { return rng_->unirand(a, b); }
	// device
	int device_ = 0;
	cudaStream_t stream_ = nullptr;
	bool own_stream_ = false;
	float2* d_pgr_ = nullptr;      // phase gratings [sum nvar][npgy][npgx]
	float2* d_pro_ = nullptr;      // propagators [npro][ny][nx]
	float* d_det_ = nullptr;       // detector functions with masks folded in [ndet][ny][nx]
	float2* d_wav0_ = nullptr;     // incident wave backup
	float2* d_wav_ = nullptr;      // offset wave (input of GPUMultislice)
	float* d_cppl_ = nullptr;      // constant phase plate
	float2* d_twx_ = nullptr;      // twiddles exp(-2 pi i k/nx)
	float2* d_twy_ = nullptr;
	float2* d_work_ = nullptr;     // working waves [nwave][ny][nx]
	size_t work_cap_ = 0;          // capacity in complex elements
	float* d_partial_ = nullptr;   // per-CTA detector partial sums
	size_t partial_cap_ = 0;
	double* d_detint_ = nullptr;   // single-run integrated detectors [ndetslc][ndet]
	double* d_shift_ = nullptr;    // per-wave offsets (scan)
	size_t shift_cap_ = 0;
	float *d_dif_ = nullptr, *d_img_ = nullptr, *d_dif_avg_ = nullptr, *d_img_avg_ = nullptr;
	float2 *d_wff_ = nullptr, *d_wfr_ = nullptr, *d_wff_avg_ = nullptr, *d_wfr_avg_ = nullptr;
	float weight_imgavg_ = 0.f, weight_wavavg_ = 0.f;
	int scan_batch_ = 32;
	int descan_on_ = 0, descan_x_ = 0, descan_y_ = 0;
	int timing_on_ = 0;
	const PlanOps* prow_ = nullptr;  // plan of the row / entry passes (length nx)
	const PlanOps* pcol_ = nullptr;  // plan of the column / exit passes (length ny)
	std::vector<cudaEvent_t> ev_col_, ev_row_;   // start/stop pairs
	cudaEvent_t timed_event();
	int plasmon_on_ = 0;
	float pl_qe_ = 0.f, pl_qc_ = 0.f, pl_mfp_ = 0.f;
	unsigned int pl_nmax_ = 0, pl_nex_ = 0;
	float pl_tqx_ = 0.f, pl_tqy_ = 0.f;
	int* d_plas_ = nullptr;         // per-wave plasmon shifts of a scan chunk [nobj][nwave][2]
	size_t plas_cap_ = 0;
	long long launches_ = 0;
	int prec_ = 0;                  // 0 FP32, 1 BF16 hi+lo tensor core, 2 FP16 hi+lo tensor core
	int* d_tcerr_ = nullptr;        // tensor-core pass status word
	long long tc_launches_ = 0;
	double* d_scratch_ = nullptr;
	size_t scratch_cap_ = 0;
	double* d_cv_ = nullptr;        // CvScratch: two halves of 2 n doubles
	size_t cv_cap_ = 0;             // n of the current buffer
	int cv_half_ = 0;
	cudaEvent_t cv_done_[2] = {nullptr, nullptr};
	int fuse_passes_ = 1;
	int* d_mulw_ = nullptr;         // per-slice per-wave grating offsets of a fused scan launch
	size_t mulw_cap_ = 0;
	double* d_shiftw_ = nullptr;    // per-wave probe offsets of a fused scan launch
	size_t shiftw_cap_ = 0;
	std::vector<int> h_mulw_;
	uint8_t* d_io_ = nullptr;       // ScanGPU's device staging (positions, sums, binned patterns)
	size_t io_cap_ = 0;
	cudaError_t last_cuda_ = cudaSuccess;
};

} // namespace jms
