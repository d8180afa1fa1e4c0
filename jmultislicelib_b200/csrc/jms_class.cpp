// jms_class.cpp -- the C++ class interface (include/JMultiSlice.h,
// include/JProbeGen.h, include/rng.h) over the library's context class.
//
// CJMultiSlice (src/JMultiSlice.h:403-936) owns one jms::JmsB200, the same
// context class that serves the flat C interface, made on the first call so
// that a static CJMultiSlice costs nothing before it is used.  Every method
// forwards with the reference's argument meaning; fcmplx arrays are passed on
// as interleaved float pairs, which is their memory layout.
#include "../../include/JMultiSlice.h"
#include "jms_host.h"

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <thread>

// ---------------------------------------------------------------------------
// CRng (src/rng.h:30-65): the reference's draw formulas on std::mt19937
// ---------------------------------------------------------------------------
CRng::CRng() : uni_dist(0, RAND_MAXROLL), norm_dist(0.0, 1.0), m_seed((int)std::time(nullptr))
{
	urng.seed((std::mt19937::result_type)m_seed);
}

CRng::CRng(int seed) : uni_dist(0, RAND_MAXROLL), norm_dist(0.0, 1.0), m_seed(seed)
{
	urng.seed((std::mt19937::result_type)m_seed);
}

CRng::~CRng() {}

void CRng::seed(int seed)
{
	m_seed = (seed == 0) ? (int)std::time(nullptr) : seed;
	urng.seed((std::mt19937::result_type)m_seed);
}

int CRng::get_seed(void) { return m_seed; }

int CRng::rand() { return uni_dist(urng); }

double CRng::unirand(double rmin, double rmax)
{
	return rmin + ((double)rand() / (double)((unsigned long)RAND_MAXROLL)) * (rmax - rmin);
}

double CRng::unirand_oub(double rmin, double rmax)
{
	return rmin + ((double)rand() / (double)((unsigned long)RAND_MAXROLL + 1)) * (rmax - rmin);
}

double CRng::normrand(double mu, double sdev) { return mu + sdev * norm_dist(urng); }

int CRng::poisrand(double mu)
{
	std::poisson_distribution<int> pd(mu);
	return pd(urng);
}

// ---------------------------------------------------------------------------
// CJProbeParams (src/JProbeGen.h:60-140, defaults src/JProbeGen.cpp:53-80)
// ---------------------------------------------------------------------------
namespace {
// aberrations up to order o: sum over orders of the rotational symmetries
// (src/JProbeGen.cpp:60-61 counts them in closed form); 24 for order 8
int aberration_count(int omax)
{
	int n = 0;
	for (int o = 1; o <= omax; o++) n += o / 2 + 1;
	return n;
}

void probe_defaults(CJProbeParams& p)
{
	p.m_wl = 0.001969f;
	p.m_alpha = 0.025f;
	p.m_alpha_rs = 0.03f;
	p.m_alpha_x0 = p.m_alpha_y0 = 0.f;
	p.m_alpha_asym = p.m_alpha_adir = 0.f;
	p.m_btx = p.m_bty = 0.f;
	p.m_source_width = 0.f;
	p.m_source_shape = 0;
	p.m_fspread_width = 0.f;
	p.m_fspread_kernel_width = 2.f;
	p.m_fspread_kernel_samples = 7;
}

void probe_copy_data(CJProbeParams& d, const CJProbeParams& s)
{
	d.m_wl = s.m_wl;
	d.m_alpha = s.m_alpha;
	d.m_alpha_rs = s.m_alpha_rs;
	d.m_alpha_x0 = s.m_alpha_x0;
	d.m_alpha_y0 = s.m_alpha_y0;
	d.m_alpha_asym = s.m_alpha_asym;
	d.m_alpha_adir = s.m_alpha_adir;
	d.m_btx = s.m_btx;
	d.m_bty = s.m_bty;
	d.m_source_width = s.m_source_width;
	d.m_source_shape = s.m_source_shape;
	d.m_fspread_width = s.m_fspread_width;
	d.m_fspread_kernel_width = s.m_fspread_kernel_width;
	d.m_fspread_kernel_samples = s.m_fspread_kernel_samples;
}
} // namespace

CJProbeParams::CJProbeParams(void)
{
	m_abrr_num = aberration_count(_JPG_ABERRATION_ORDER_MAX);
	m_abrr_coeff = (float*)std::calloc((size_t)2 * m_abrr_num, sizeof(float));
	m_msg[0] = 0;
	probe_defaults(*this);
}

CJProbeParams::CJProbeParams(const CJProbeParams& src)
{
	m_abrr_num = aberration_count(_JPG_ABERRATION_ORDER_MAX);
	m_abrr_coeff = (float*)std::calloc((size_t)2 * m_abrr_num, sizeof(float));
	m_msg[0] = 0;
	probe_copy_data(*this, src);
	const int n = 2 * std::min(m_abrr_num, const_cast<CJProbeParams&>(src).GetAberrationNum());
	if (m_abrr_coeff && src.m_abrr_coeff && n > 0) std::memcpy(m_abrr_coeff, src.m_abrr_coeff, sizeof(float) * n);
}

CJProbeParams::~CJProbeParams(void)
{
	std::free(m_abrr_coeff);
}

void CJProbeParams::operator=(const CJProbeParams& other)
{
	probe_copy_data(*this, other);
	const int n = 2 * std::min(m_abrr_num, const_cast<CJProbeParams&>(other).GetAberrationNum());
	if (m_abrr_coeff && other.m_abrr_coeff && n > 0) std::memcpy(m_abrr_coeff, other.m_abrr_coeff, sizeof(float) * n);
}

bool CJProbeParams::operator==(const CJProbeParams& o) const
{
	if (m_abrr_num != const_cast<CJProbeParams&>(o).GetAberrationNum()) return false;
	return m_wl == o.m_wl && m_alpha == o.m_alpha && m_alpha_rs == o.m_alpha_rs && m_alpha_x0 == o.m_alpha_x0 &&
		m_alpha_y0 == o.m_alpha_y0 && m_alpha_asym == o.m_alpha_asym && m_alpha_adir == o.m_alpha_adir &&
		m_btx == o.m_btx && m_bty == o.m_bty && m_source_width == o.m_source_width &&
		m_source_shape == o.m_source_shape && m_fspread_width == o.m_fspread_width &&
		m_fspread_kernel_width == o.m_fspread_kernel_width && m_fspread_kernel_samples == o.m_fspread_kernel_samples &&
		std::memcmp(m_abrr_coeff, o.m_abrr_coeff, sizeof(float) * 2 * m_abrr_num) == 0;
}

int CJProbeParams::GetAberrationNum(void) { return m_abrr_num; }

float CJProbeParams::SetProbeEkV(float ekv)
{
	m_wl = jms::wavelength_nm(ekv);
	return m_wl;
}

// ---------------------------------------------------------------------------
// CJMultiSlice
// ---------------------------------------------------------------------------
CJMultiSlice::CJMultiSlice() : m_impl(nullptr), m_dbg(0) { m_msg[0] = 0; }

CJMultiSlice::~CJMultiSlice() { delete m_impl; }

jms::JmsB200* CJMultiSlice::Context(void)
{
	if (m_impl == nullptr) m_impl = new jms::JmsB200();
	return m_impl;
}

int CJMultiSlice::SetDebugLevel(int dbg)
{
	const int o = m_dbg;
	m_dbg = dbg;
	return o;
}

int CJMultiSlice::Cleanup(void) { return Context()->Cleanup(); }
void CJMultiSlice::FreeLibMem(void) {}   // no FFT library state to release
float CJMultiSlice::SetHighTension(float ht) { return Context()->SetHighTension(ht); }
void CJMultiSlice::SetSupercellSize(float* a0) { if (a0) Context()->SetSupercellSize(a0[0], a0[1], a0[2]); }
void CJMultiSlice::SetSupercellSize(float a, float b, float c) { Context()->SetSupercellSize(a, b, c); }
void CJMultiSlice::SetGridSize(int nx, int ny) { Context()->SetGridSize(nx, ny); }
void CJMultiSlice::SetSliceThickness(int islc, float t) { Context()->SetSliceThickness(islc, t); }

int CJMultiSlice::SetDetectionPlanes(int ndetper, int nobjslc, int* det_objslc)
{
	return Context()->SetDetectionPlanes(ndetper, nobjslc, det_objslc);
}

int CJMultiSlice::SetDetectionPlanes(std::vector<int> slc_det, int nobjslc, int* det_objslc)
{
	return Context()->SetDetectionPlanesList(slc_det.data(), (int)slc_det.size(), nobjslc, det_objslc);
}

void CJMultiSlice::SetPlasmonMC(bool use, float q_e, float q_c, float mfp, unsigned int nexmax)
{
	Context()->SetPlasmonMC(use, q_e, q_c, mfp, nexmax);
}
void CJMultiSlice::DiffractionDescan(bool on) { Context()->DiffractionDescan(on); }
void CJMultiSlice::SetDiffractionDescanN(int whichcode, int ndx, int ndy, int)
{ Context()->SetDiffractionDescanN(whichcode, ndx, ndy); }
void CJMultiSlice::SetDiffractionDescan(int whichcode, float dx, float dy, int)
{ Context()->SetDiffractionDescan(whichcode, dx, dy); }
void CJMultiSlice::SetDiffractionDescanMRad(int whichcode, float dx, float dy, int)
{ Context()->SetDiffractionDescanMRad(whichcode, dx, dy); }

int CJMultiSlice::CalculateProbeWaveFourier(CJProbeParams* prm, fcmplx* wav)
{
	if (prm == nullptr || wav == nullptr) return 1;
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
	const int n = std::min(2 * prm->GetAberrationNum(), (int)(sizeof(p.abrr) / sizeof(float)));
	if (prm->m_abrr_coeff && n > 0) std::memcpy(p.abrr, prm->m_abrr_coeff, sizeof(float) * n);
	return Context()->CalculateProbeWaveFourier(p, reinterpret_cast<float*>(wav));
}

int CJMultiSlice::CalculatePropagator(float fthick, float otx, float oty, fcmplx* pro, int ntype)
{
	return Context()->CalculatePropagator(fthick, otx, oty, reinterpret_cast<float*>(pro), ntype);
}

int CJMultiSlice::CalculateRingDetector(float beta0, float beta1, float phi0, float phi1, float theta0x,
	float theta0y, std::string sdsprofile, float* det, int& msklen, int* msk, int kmom1)
{
	return Context()->CalculateRingDetector(beta0, beta1, phi0, phi1, theta0x, theta0y, sdsprofile.c_str(), det,
		&msklen, msk, kmom1);
}

int CJMultiSlice::PhaseGratingSetup(int whichcode, int nx, int ny, int nslc, int nvarmax, int* nslcvar)
{ return Context()->PhaseGratingSetup(whichcode, nx, ny, nslc, nvarmax, nslcvar); }
int CJMultiSlice::ObjectSliceSetup(int nobjslc, int* objslc) { return Context()->ObjectSliceSetup(nobjslc, objslc); }
int CJMultiSlice::PropagatorSetup(int whichcode, int npro, int* proidx)
{ return Context()->PropagatorSetup(whichcode, npro, proidx); }
int CJMultiSlice::DetectorSetup(int whichcode, int ndetper, int ndetint, int imagedet, int nthreads_CPU)
{ return Context()->DetectorSetup(whichcode, ndetper, ndetint, imagedet, nthreads_CPU); }
int CJMultiSlice::DetectorSetup(int whichcode, std::vector<int> slc_det, int ndetint, int imagedet, int nthreads_CPU)
{
	return Context()->DetectorSetupList(whichcode, slc_det.data(), (int)slc_det.size(), ndetint, imagedet,
		nthreads_CPU);
}
int CJMultiSlice::SetPhaseGratingData(int whichcode, int islc, int nvar, fcmplx* pgr)
{ return Context()->SetPhaseGratingData(whichcode, islc, nvar, reinterpret_cast<const float*>(pgr)); }
int CJMultiSlice::SetPropagatorData(int whichcode, int ipro, fcmplx* pro)
{ return Context()->SetPropagatorData(whichcode, ipro, reinterpret_cast<const float*>(pro)); }
int CJMultiSlice::SetDetectorData(int whichcode, int idet, float* det, int msklen, int* msk)
{ return Context()->SetDetectorData(whichcode, idet, det, msklen, msk); }
int CJMultiSlice::InitCore(int whichcode, int nCPUthreads) { return Context()->InitCore(whichcode, nCPUthreads); }
int CJMultiSlice::SetIncidentWave(int whichcode, fcmplx* wav, bool bTranspose)
{ return Context()->SetIncidentWave(whichcode, reinterpret_cast<const float*>(wav), bTranspose); }
int CJMultiSlice::SetIncidentWavePhaseplate(int whichcode, float* ppl, bool bTranspose)
{ return Context()->SetIncidentWavePhaseplate(whichcode, ppl, bTranspose); }
int CJMultiSlice::ZeroIncidentWavePhaseplate(int whichcode) { return Context()->ZeroIncidentWavePhaseplate(whichcode); }
int CJMultiSlice::GetUnscrambleHash(unsigned int* phash) { return Context()->GetUnscrambleHash(phash); }
int CJMultiSlice::GetDetetionSliceNum(void) { return Context()->GetDetetionSliceNum(); }
int CJMultiSlice::GetDetNum(void) { return Context()->GetDetNum(); }
float CJMultiSlice::GetHighTension(void) { return Context()->GetHighTension(); }
float CJMultiSlice::GetWaveLength(void) { return Context()->GetWaveLength(); }
void CJMultiSlice::GetGridSize(int& nx, int& ny) { Context()->GetGridSize(nx, ny); }
void CJMultiSlice::GetSupercellSize(float* a0) { if (a0) Context()->GetSupercellSize(a0); }
void CJMultiSlice::GetSupercellSize(float& a, float& b, float& c)
{
	float a0[3];
	Context()->GetSupercellSize(a0);
	a = a0[0];
	b = a0[1];
	c = a0[2];
}
float CJMultiSlice::GetSliceThickness(int islc) { return Context()->GetSliceThickness(islc); }

int CJMultiSlice::GetCPUNum(void) { return (int)std::thread::hardware_concurrency(); }
int CJMultiSlice::GetJCPUcorenum(void) { return 0; }   // no CPU calculation threads
int CJMultiSlice::GetGPUNum(void)
{
	int n = 0;
	return cudaGetDeviceCount(&n) == cudaSuccess ? n : 0;
}
int CJMultiSlice::GetGPUName(int idev, char* name)
{
	cudaDeviceProp p;
	if (name == nullptr || cudaGetDeviceProperties(&p, idev) != cudaSuccess) return 1;
	std::strncpy(name, p.name, 255);
	name[255] = 0;
	return 0;
}
int CJMultiSlice::GetCurrentGPU(void) { return Context()->GetCurrentGPU(); }
int CJMultiSlice::SetCurrentGPU(int idev) { return Context()->SetCurrentGPU(idev); }
int CJMultiSlice::GetGPUStats(int idev, int& iCMajor, int& iCMinor, int& iMaxThread, int64_t& memtotal,
	int64_t& memfree)
{
	cudaDeviceProp p;
	if (cudaGetDeviceProperties(&p, idev) != cudaSuccess) return 1;
	iCMajor = p.major;
	iCMinor = p.minor;
	iMaxThread = p.maxThreadsPerBlock;
	int cur = 0;
	size_t f = 0, t = 0;
	cudaGetDevice(&cur);
	cudaSetDevice(idev);
	const cudaError_t e = cudaMemGetInfo(&f, &t);
	cudaSetDevice(cur);
	memtotal = (int64_t)t;
	memfree = (int64_t)f;
	return e == cudaSuccess ? 0 : 2;
}
int CJMultiSlice::GetGPUMemInfo(size_t& memtotal, size_t& memfree)
{
	return cudaMemGetInfo(&memfree, &memtotal) == cudaSuccess ? 0 : 1;
}
int CJMultiSlice::SetGPUPgrLoading(int npgrload) { return Context()->SetGPUPgrLoading(npgrload); }
void CJMultiSlice::SetRng(CRng* prng) { Context()->SetRng(prng); }
CRng* CJMultiSlice::GetRng(void) { return Context()->GetRng(); }
void CJMultiSlice::SeedRngEx(int nseed) { Context()->SeedRngEx(nseed); }
int CJMultiSlice::ClearDetMem_h(int) { return 1; }
int CJMultiSlice::ClearDetMem_d(void) { return Context()->ClearDetMem_d(); }

int CJMultiSlice::OffsetIncomingWave(int whichcode, float dx, float dy, float dz, int iThread, int ibtx, int ibty,
	bool bcppl)
{ return Context()->OffsetIncomingWave(whichcode, dx, dy, dz, iThread, ibtx, ibty, bcppl); }
int CJMultiSlice::SetIncomingWaveGPU(fcmplx* wav, bool bTranspose)
{ return Context()->SetIncomingWaveGPU(reinterpret_cast<const float*>(wav), bTranspose); }
int CJMultiSlice::SetIncomingWaveCPU(fcmplx*, bool, int) { return 1; }
int CJMultiSlice::CPUMultislice(int, int, float, int) { return 1; }
int CJMultiSlice::GPUMultislice(int islc0, int accmode, float weight)
{ return Context()->GPUMultislice(islc0, accmode, weight); }
int CJMultiSlice::GetResult(int whichcode, int whichresult, float* dst, int iThread)
{ return Context()->GetResult(whichcode, whichresult, dst, iThread); }
int CJMultiSlice::GetAvgResult(int whichcode, int whichresult, float* dst, float& weight, int iThread)
{ return Context()->GetAvgResult(whichcode, whichresult, dst, &weight, iThread); }
float CJMultiSlice::GetImageAveragingWeight(int whichcode, int iThread)
{ return Context()->GetImageAveragingWeight(whichcode, iThread); }
float CJMultiSlice::GetWaveAveragingWeight(int whichcode, int iThread)
{ return Context()->GetWaveAveragingWeight(whichcode, iThread); }
int CJMultiSlice::ResetImageAveraging(int whichcode, int iThread)
{ return Context()->ResetImageAveraging(whichcode, iThread); }
int CJMultiSlice::ResetWaveAveraging(int whichcode, int iThread)
{ return Context()->ResetWaveAveraging(whichcode, iThread); }
int CJMultiSlice::ReadoutDetAvg(int whichcode, int whichresult, float* dst, float& weight, int iThread)
{ return Context()->ReadoutDetAvg(whichcode, whichresult, dst, &weight, iThread); }
int CJMultiSlice::GetRandomVariantSequence(int* out) { return Context()->GetRandomVariantSequence(out); }
