// jms_capi.cpp -- flat C interface (include/jms_b200.h) over one library
// instance, as JMultiSliceLib.cpp forwards to its static CJMultiSlice
// (src/JMultiSliceLib.h:106, src/JMultiSliceLib.cpp).
#include "../../include/jms_b200.h"
#include "jms_host.h"
#include "jms_kernels.h"
#include "jms_pgr_host.h"

#include <cstdio>
#include <cstring>
#include <memory>
#include <thread>
#include <vector>

using jms::JmsB200;

static JmsB200& J()
{
	static std::unique_ptr<JmsB200> inst(new JmsB200());
	return *inst;
}

static jms::PgrGen& G()
{
	static std::unique_ptr<jms::PgrGen> inst(new jms::PgrGen());
	return *inst;
}

static int g_debug = 0;

extern "C" {

float GetJMSVersion(void) { return 0.46f; }
int SetJMSDebugLevel(int debuglevel) { int o = g_debug; g_debug = debuglevel; return o; }
void SeedRngEx(int rngseed) { J().SeedRngEx(rngseed); }

float SetHighTension(float ht) { return J().SetHighTension(ht); }
float GetHighTension(void) { return J().GetHighTension(); }
float GetWaveLength(void) { return J().GetWaveLength(); }
void SetSupercellSize(float* a0) { if (a0) J().SetSupercellSize(a0[0], a0[1], a0[2]); }
void SetSupercellSizeABC(float a, float b, float c) { J().SetSupercellSize(a, b, c); }
void SetSliceThickness(int islc, float fthickness) { J().SetSliceThickness(islc, fthickness); }
void DiffractionDescan(int bActivate) { J().DiffractionDescan(bActivate != 0); }
void SetPlasmonMC(int bActivate, float fq_e, float fq_c, float fmfp, unsigned int nexmax)
{ J().SetPlasmonMC(bActivate != 0, fq_e, fq_c, fmfp, nexmax); }
void SetDiffractionDescanN(int whichcode, int ndescanx, int ndescany, int) { J().SetDiffractionDescanN(whichcode, ndescanx, ndescany); }
void SetDiffractionDescan(int whichcode, float descanx, float descany, int) { J().SetDiffractionDescan(whichcode, descanx, descany); }
void SetDiffractionDescanMRad(int whichcode, float descanx, float descany, int) { J().SetDiffractionDescanMRad(whichcode, descanx, descany); }

void SetGridSize(int nx, int ny) { J().SetGridSize(nx, ny); }
void GetGridSize(int* nx, int* ny) { int a = 0, b = 0; J().GetGridSize(a, b); if (nx) *nx = a; if (ny) *ny = b; }
int GetDetetionSliceNum(void) { return J().GetDetetionSliceNum(); }
int GetDetNum(void) { return J().GetDetNum(); }
int GetCPUNum(void) { return (int)std::thread::hardware_concurrency(); }
int GetGPUNum(void) { int n = 0; if (cudaGetDeviceCount(&n) != cudaSuccess) return 0; return n; }
int GetGPUName(int idev, char* name)
{
	cudaDeviceProp p;
	if (!name || cudaGetDeviceProperties(&p, idev) != cudaSuccess) return 1;
	std::strncpy(name, p.name, 255);
	name[255] = 0;
	return 0;
}
int GetCurrentGPU(void) { return J().GetCurrentGPU(); }
int SetCurrentGPU(int idev) { return J().SetCurrentGPU(idev); }
int GetGPUStats(int idev, int* iCMajor, int* iCMinor, int* iMaxThread, int64_t* memtotal, int64_t* memfree)
{
	cudaDeviceProp p;
	if (cudaGetDeviceProperties(&p, idev) != cudaSuccess) return 1;
	if (iCMajor) *iCMajor = p.major;
	if (iCMinor) *iCMinor = p.minor;
	if (iMaxThread) *iMaxThread = p.maxThreadsPerBlock;
	size_t f = 0, t = 0;
	int cur = 0;
	cudaGetDevice(&cur);
	cudaSetDevice(idev);
	cudaMemGetInfo(&f, &t);
	cudaSetDevice(cur);
	if (memtotal) *memtotal = (int64_t)t;
	if (memfree) *memfree = (int64_t)f;
	return 0;
}
int GetUnscrambleHash(unsigned int* phash) { return J().GetUnscrambleHash(phash); }
float GetImageAveragingWeight(int whichcode, int iThread) { return J().GetImageAveragingWeight(whichcode, iThread); }
float GetWaveAveragingWeight(int whichcode, int iThread) { return J().GetWaveAveragingWeight(whichcode, iThread); }

int PhaseGratingSetup(int whichcode, int nx, int ny, int nslc, int nvarmax, int* nslcvar)
{ return J().PhaseGratingSetup(whichcode, nx, ny, nslc, nvarmax, nslcvar); }
int ObjectSliceSetup(int nobjslc, int* objslc) { return J().ObjectSliceSetup(nobjslc, objslc); }
int PropagatorSetup(int whichcode, int npro, int* proidx) { return J().PropagatorSetup(whichcode, npro, proidx); }
int DetectorSetup(int whichcode, int ndetper, int ndetint, int imagedet, int nthreads_CPU)
{ return J().DetectorSetup(whichcode, ndetper, ndetint, imagedet, nthreads_CPU); }
int InitCore(int whichcode, int nCPUthreads) { return J().InitCore(whichcode, nCPUthreads); }
int SetIncidentWave(int whichcode, float* wav) { return J().SetIncidentWave(whichcode, wav, false); }
int SetIncidentWavePhaseplate(int whichcode, float* ppl, int bTranspose)
{ return J().SetIncidentWavePhaseplate(whichcode, ppl, bTranspose != 0); }
int ZeroIncidentWavePhaseplate(int whichcode) { return J().ZeroIncidentWavePhaseplate(whichcode); }
int SetSlicePhaseGratings(int whichcode, int islc, int nvar, float* pgr)
{ return J().SetPhaseGratingData(whichcode, islc, nvar, pgr); }
int SetPropagatorData(int whichcode, int ipro, float* pro) { return J().SetPropagatorData(whichcode, ipro, pro); }
int SetDetectorData(int whichcode, int idet, float* det, int msklen, int* msk)
{ return J().SetDetectorData(whichcode, idet, det, msklen, msk); }
int SetGPUPgrLoading(int npgrload) { return J().SetGPUPgrLoading(npgrload); }
int ResetImageAveraging(int whichcode, int iThread) { return J().ResetImageAveraging(whichcode, iThread); }
int ResetWaveAveraging(int whichcode, int iThread) { return J().ResetWaveAveraging(whichcode, iThread); }

int CalculateProbeWaveFourier(JMSProbeParams* prm, float* wav)
{
	if (!prm || !wav) return 1;
	jms::ProbeParams p;
	p.wl = prm->m_wl;
	p.alpha = prm->m_alpha;
	p.alpha_rs = prm->m_alpha_rs;
	p.alpha_x0 = prm->m_alpha_x0;
	p.alpha_y0 = prm->m_alpha_y0;
	p.alpha_asym = prm->m_alpha_asym;
	p.alpha_adir = prm->m_alpha_adir;
	p.btx = prm->m_btx;
	p.bty = prm->m_bty;
	if (prm->m_abrr_coeff) std::memcpy(p.abrr, prm->m_abrr_coeff, sizeof(p.abrr));
	return J().CalculateProbeWaveFourier(p, wav);
}
int SetIncomingWaveGPU(float* wav, int bTranspose) { return J().SetIncomingWaveGPU(wav, bTranspose != 0); }
int SetIncomingWaveCPU(float*, int, int) { return 1; }
int CalculatePropagator(float fthick, float otx, float oty, float* pro, int ntype)
{ return J().CalculatePropagator(fthick, otx, oty, pro, ntype); }
int CalculateRingDetector(float beta0, float beta1, float phi0, float phi1, float theta0x, float theta0y,
	const char* sdsprofile, float* det, int* msklen, int* msk, int kmom1)
{
	// the reference's flat interface passes theta0x twice (src/JMultiSliceLib.cpp:254);
	// here theta0y reaches the class as intended
	return J().CalculateRingDetector(beta0, beta1, phi0, phi1, theta0x, theta0y, sdsprofile, det, msklen, msk, kmom1);
}
int OffsetIncomingWave(int whichcode, float dx, float dy, float dz, int iThread, int ibtx, int ibty)
{ return J().OffsetIncomingWave(whichcode, dx, dy, dz, iThread, ibtx, ibty, true); }
int CPUMultislice(int, int, float, int) { return 1; }
int GPUMultislice(int islc0, int accmode, float weight) { return J().GPUMultislice(islc0, accmode, weight); }
int GetResult(int whichcode, int whichresult, float* dst, int iThread)
{ return J().GetResult(whichcode, whichresult, dst, iThread); }
int GetAvgResult(int whichcode, int whichresult, float* dst, float* wgt, int iThread)
{ return J().GetAvgResult(whichcode, whichresult, dst, wgt, iThread); }
int ClearDetMem_h(int) { return 1; }
int ClearDetMem_d(void) { return J().ClearDetMem_d(); }
int Cleanup(void) { return J().Cleanup(); }
void FreeLibMem(void) {}

int JMS_SetStream(void* stream) { return J().SetStream((cudaStream_t)stream); }
int JMS_ScanGPU(int npos, const float* pos, float dz, int npass, const int* varseq, float* out_int, float* out_bin,
	int bin)
{ return J().ScanGPU(npos, pos, dz, npass, varseq, out_int, out_bin, bin); }
int JMS_ScanGPUDevice(int npos, const float* d_pos, float dz, int npass, const int* varseq, double* d_out_int,
	float* d_out_bin, int bin)
{ return J().ScanGPUDevice(npos, d_pos, dz, npass, varseq, d_out_int, d_out_bin, bin); }
int JMS_SetScanBatch(int nwave) { return J().SetScanBatch(nwave); }
long long JMS_KernelLaunches(void) { return J().KernelLaunches(); }
void JMS_SetPassTiming(int on) { J().SetPassTiming(on); }
int JMS_PassTiming(double* ms_col, long long* n_col, double* ms_row, long long* n_row)
{ return J().PassTiming(ms_col, n_col, ms_row, n_row); }
int JMS_ReadoutDetectorsNoAlloc(const float* d_wav, int nwave, double* d_out, void* stream)
{ return J().ReadoutDetectorsNoAlloc(d_wav, nwave, d_out, (cudaStream_t)stream); }
int JMS_Autotune(int nwave, int reps, float* ms_row, float* ms_col, int* irow, int* icol)
{ return J().Autotune(nwave, reps, ms_row, ms_col, irow, icol); }
int JMS_SelectPlans(int irow, int icol) { return J().SelectPlans(irow, icol); }
int JMS_PlanCount(int n) { return jms::plan_count(n); }
int JMS_PlanName(int axis, char* name, int len)
{
	if (!name || len < 1) return 1;
	std::strncpy(name, J().PlanName(axis), (size_t)len - 1);
	name[len - 1] = 0;
	return 0;
}
int JMS_GridSupported(int nx, int ny) { return (jms::pass_supported(nx) && jms::pass_supported(ny)) ? 1 : 0; }

int JMS_ReadoutDetAvg(int whichcode, int whichresult, float* dst, float* weight)
{ return J().ReadoutDetAvg(whichcode, whichresult, dst, weight, 0); }

int JMS_SliLoadSlice(const char* path, int islc)
{
	JMSSliHeader h;
	int e = JMS_SliReadHeader(path, &h);
	if (e) return e;
	int npgx = 0, npgy = 0;
	if (J().GratingSlot(islc, 0, 1, &npgx, &npgy) == nullptr) return 1;
	if (h.nx != npgx || h.ny != npgy) return 7;
	std::vector<float> buf((size_t)2 * h.nx * h.ny * h.nvar);
	if ((e = JMS_SliReadData(path, buf.data()))) return e;
	return J().SetPhaseGratingData(jms::CODE_GPU, islc, h.nvar, buf.data());
}

int JMS_PgrSetup(int nx, int ny, float a, float b, float ekv, int thermal, int bwl_pot, int bwl_pgr)
{
	G().Reset();
	int e = G().SetGrid(nx, ny, a, b);
	if (e) return e;
	return G().SetPhysics(ekv, thermal, bwl_pot, bwl_pgr);
}
int JMS_PgrSetFormFactors(int ntype, int nk, float sk, const float* ff, const float* biso)
{ return G().SetFormFactors(ntype, nk, sk, ff, biso); }
int JMS_PgrCalculate(int natom, const float* atoms, float cz, int ngr, unsigned long long seed, int islc, int ivar0,
	float* pgr)
{
	float2* dst = nullptr;
	if (islc >= 0) {
		int npgx = 0, npgy = 0;
		dst = J().GratingSlot(islc, ivar0, ngr, &npgx, &npgy);
		if (dst == nullptr || npgx != G().nx() || npgy != G().ny()) return 9;
	}
	G().SetStream(J().Stream());
	return G().Calculate(natom, atoms, cz, ngr, seed, dst, pgr);
}

} // extern "C"
