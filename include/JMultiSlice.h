/*
 * JMultiSlice.h -- C++ class interface of the B200 multislice library.
 *
 * Declares class CJMultiSlice with the public methods, overloads and default
 * arguments of the reference class (src/JMultiSlice.h:403-936), so that code
 * written against the reference's header compiles unchanged against this one
 * and runs on libjms_b200.so.  The reference's calling order holds
 * (src/JMultiSlice.h:77-97):
 *   SetHighTension, SetGridSize, SetSupercellSize;
 *   PhaseGratingSetup, ObjectSliceSetup, PropagatorSetup, DetectorSetup;
 *   SetPhaseGratingData, SetPropagatorData, SetDetectorData;
 *   InitCore, SetIncidentWave;
 *   then per run OffsetIncomingWave, GPUMultislice, GetResult.
 *
 * One object is one library context: its own grid, setup, device buffers and
 * CUDA stream (created by InitCore on the current device).  Objects are
 * independent, so several of them (different grids, different devices) can
 * live in one process.  A single object's GPU calls are not re-entrant, as in
 * the reference.  The object is created without touching the GPU; its
 * context is made on the first call.
 *
 * Differences from the reference, all in what the reference computes on the
 * CPU:
 *   - there is no CPU code path.  Calls whose whichcode has the _JMS_CODE_CPU
 *     bit set return 1 and do nothing (CPUMultislice, SetIncomingWaveCPU and
 *     ClearDetMem_h always do);
 *   - SetGPUPgrLoading is accepted, but phase gratings always stay in device
 *     memory (the reference's on-demand upload exists to save memory on
 *     small GPUs);
 *   - the protected helpers of the reference's CPU path and memory handling
 *     (DotProduct_h, AllocMem_h, GetPhaseGrating_h, ...) are not declared.
 *
 * Complex arrays are fcmplx = std::complex<float>, row-major [ny][nx] with x
 * fastest, Fourier space in scrambled (FFT) order, as in the reference.
 * Results: integrated detectors [ndetslc][ndet] (GetResult with
 * _JMS_DETECT_INTEGRATED), images and diffraction patterns [ndetslc][ny][nx],
 * waves [ndetslc][ny][nx] complex.  Error codes are the reference's.
 */
#ifndef JMS_B200_JMULTISLICE_H
#define JMS_B200_JMULTISLICE_H

#include <complex>
#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include "JProbeGen.h"
#include "rng.h"

typedef std::complex<float> fcmplx;

/* version of the reference interface this class follows */
#define __JMS_VERSION__          0
#define __JMS_VERSION_SUB__      4
#define __JMS_VERSION_SUB_SUB__  5
/* code ids */
#define _JMS_CODE_CPU            1
#define _JMS_CODE_GPU            2
/* setup status bits and thresholds */
#define _JMS_STATUS_NONE         0
#define _JMS_STATUS_PGR          1
#define _JMS_STATUS_OBJ          2
#define _JMS_STATUS_PRO          4
#define _JMS_STATUS_DET          8
#define _JMS_STATUS_CORE         16
#define _JMS_THRESHOLD_CORE      15
#define _JMS_THRESHOLD_CALC      31
/* accumulation and detection flags */
#define _JMS_ACCMODE_NONE        0
#define _JMS_ACCMODE_INTEGRATE   1
#define _JMS_DETECT_NONE         0
#define _JMS_DETECT_INTEGRATED   1
#define _JMS_DETECT_IMAGE        2
#define _JMS_DETECT_DIFFRACTION  4
#define _JMS_DETECT_WAVEREAL     8
#define _JMS_DETECT_WAVEFOURIER  16
#define _JMS_DETECT_IMAGE_AVG    32
#define _JMS_DETECT_DIFFR_AVG    64
#define _JMS_DETECT_WAVER_AVG    128
#define _JMS_DETECT_WAVEF_AVG    256
#define _JMS_MESSAGE_LEN         2048

/* relative band-width limit of the propagators */
constexpr double _JMS_RELAPERTURE = 0.666666666666667;

namespace jms { class JmsB200; }

class CJMultiSlice {
public:
	CJMultiSlice();
	~CJMultiSlice();
	CJMultiSlice(const CJMultiSlice&) = delete;
	CJMultiSlice& operator=(const CJMultiSlice&) = delete;

	/* ---- library handling and physics (src/JMultiSlice.h:403-480) ---- */
	int SetDebugLevel(int dbg);
	/* frees the setup and device memory of this object */
	int Cleanup(void);
	void FreeLibMem(void);
	/* electron energy [keV] (sets the wavelength); returns the previous energy */
	float SetHighTension(float ht);
	void SetSupercellSize(float* a0);
	void SetSupercellSize(float a, float b, float c);
	void SetGridSize(int nx, int ny);
	void SetSliceThickness(int islc, float fthickness);
	/* detection planes: every ndetper slices plus entrance and exit (period > 0),
	 * or exit only (0); det_objslc (may be NULL) receives the plane index of each
	 * object slice (-1 when none).  Returns the number of planes. */
	int SetDetectionPlanes(int ndetper, int nobjslc, int* det_objslc = NULL);
	/* the same from a list over the planes 0 .. nobjslc (0 = entrance plane):
	 * slc_det[i] >= 0 reads plane i into result index slc_det[i] */
	int SetDetectionPlanes(std::vector<int> slc_det, int nobjslc, int* det_objslc = NULL);
	/* bulk plasmon Monte-Carlo: q_e, q_c [1/nm], mean free path [nm], max. excitations */
	void SetPlasmonMC(bool use, float q_e, float q_c, float mfp, unsigned int nexmax);
	void DiffractionDescan(bool bActivate);
	void SetDiffractionDescanN(int whichcode, int ndescanx, int ndescany, int iThread = 0);
	void SetDiffractionDescan(int whichcode, float descanx, float descany, int iThread = 0);
	void SetDiffractionDescanMRad(int whichcode, float descanx, float descany, int iThread = 0);

	/* ---- generators (host, bit-identical to the reference) ---- */
	/* probe wave in Fourier space, normalised to sum |psi(k)|^2 = 1 */
	int CalculateProbeWaveFourier(CJProbeParams* prm, fcmplx* wav);
	/* propagator of slice thickness fthick [nm], object tilt (otx, oty) [mrad];
	 * ntype 0 planar (exact angles), 1 Fresnel; 2/3 band limit and 1/N included */
	int CalculatePropagator(float fthick, float otx, float oty, fcmplx* pro, int ntype = 0);
	/* annular / segmented detector [mrad, deg]; sdsprofile: sensitivity profile
	 * file ("" for none); det: function [ny][nx]; msklen / msk: the active
	 * pixels; kmom1 > 0: k-moment detector of that order */
	int CalculateRingDetector(float beta0, float beta1, float phi0, float phi1, float theta0x, float theta0y,
		std::string sdsprofile, float* det, int& msklen, int* msk = NULL, int kmom1 = 0);

	/* ---- setup chain ---- */
	int PhaseGratingSetup(int whichcode, int nx, int ny, int nslc, int nvarmax, int* nslcvar);
	int ObjectSliceSetup(int nobjslc, int* objslc);
	int PropagatorSetup(int whichcode, int npro, int* proidx);
	int DetectorSetup(int whichcode, int ndetper, int ndetint, int imagedet, int nthreads_CPU = 1);
	int DetectorSetup(int whichcode, std::vector<int> slc_det, int ndetint, int imagedet, int nthreads_CPU = 1);
	int SetPhaseGratingData(int whichcode, int islc, int nvar, fcmplx* pgr);
	int SetPropagatorData(int whichcode, int ipro, fcmplx* pro);
	int SetDetectorData(int whichcode, int idet, float* det, int msklen = 0, int* msk = NULL);
	int InitCore(int whichcode, int nCPUthreads = 1);
	int SetIncidentWave(int whichcode, fcmplx* wav, bool bTranspose = false);
	int SetIncidentWavePhaseplate(int whichcode, float* ppl, bool bTranspose = false);
	int ZeroIncidentWavePhaseplate(int whichcode);
	/* index map from scrambled to centred pixel order */
	int GetUnscrambleHash(unsigned int* phash);
	int GetDetetionSliceNum(void);
	int GetDetNum(void);
	float GetHighTension(void);
	float GetWaveLength(void);
	void GetGridSize(int& nx, int& ny);
	void GetSupercellSize(float* a0);
	void GetSupercellSize(float& a, float& b, float& c);
	float GetSliceThickness(int islc);

	/* ---- devices ---- */
	int GetCPUNum(void);
	int GetJCPUcorenum(void);
	int GetGPUNum(void);
	int GetGPUName(int idev, char* name);
	int GetCurrentGPU(void);
	/* selects the device of this object (before InitCore) */
	int SetCurrentGPU(int idev);
	int GetGPUStats(int idev, int& iCMajor, int& iCMinor, int& iMaxThread, int64_t& CUDAmemtotal,
		int64_t& CUDAmemfree);
	int GetGPUMemInfo(size_t& memtotal, size_t& memfree);
	int SetGPUPgrLoading(int npgrload = 0);
	/* random numbers of the variant draws and plasmon paths: the object's own
	 * generator (NULL) or a caller's, which must outlive the object's use */
	void SetRng(CRng* prng = NULL);
	CRng* GetRng(void);
	void SeedRngEx(int nseed = 0);

	int ClearDetMem_h(int iThread);
	int ClearDetMem_d(void);

	/* ---- calculation ---- */
	/* shifts the incident probe to (dx, dy) [nm], defocus dz [nm], beam tilt
	 * (ibtx, ibty) [pixels]; bcppl applies the constant phase plate */
	int OffsetIncomingWave(int whichcode, float dx, float dy, float dz, int iThread = 0, int ibtx = 0, int ibty = 0,
		bool bcppl = true);
	int SetIncomingWaveGPU(fcmplx* wav, bool bTranspose = false);
	int SetIncomingWaveCPU(fcmplx* wav, bool bTranspose = false, int iThread = 0);
	int CPUMultislice(int islc0, int accmode, float weight = 1.0f, int iThread = 0);
	/* multislice from object slice islc0; accmode _JMS_ACCMODE_NONE clears the
	 * detector memory first, _JMS_ACCMODE_INTEGRATE adds weight x the readouts */
	int GPUMultislice(int islc0, int accmode, float weight = 1.0f);
	int GetResult(int whichcode, int whichresult, float* dst, int iThread = 0);
	int GetAvgResult(int whichcode, int whichresult, float* dst, float& weight, int iThread = 0);
	float GetImageAveragingWeight(int whichcode, int iThread = 0);
	float GetWaveAveragingWeight(int whichcode, int iThread = 0);
	int ResetImageAveraging(int whichcode, int iThread = 0);
	int ResetWaveAveraging(int whichcode, int iThread = 0);
	/* detector readouts of the averaged waves (elastic part of a
	 * frozen-phonon average); weight receives the wave averaging weight */
	int ReadoutDetAvg(int whichcode, int whichresult, float* dst, float& weight, int iThread = 0);

	/* message buffer of the reference class (public there) */
	char m_msg[_JMS_MESSAGE_LEN];

	/* the library context behind this object (device work of the extension
	 * entry points, e.g. a batched scan) */
	jms::JmsB200* Context(void);

protected:
	/* one draw of the frozen-phonon variant of every object slice, as
	 * GPUMultislice makes it (src/JMultiSlice.cpp:1571-1676) */
	int GetRandomVariantSequence(int* out);

private:
	jms::JmsB200* m_impl;
	int m_dbg;
};

#endif /* JMS_B200_JMULTISLICE_H */
