// jms_capi.cpp -- flat C interface (include/jms_b200.h) over one library
// instance, as JMultiSliceLib.cpp forwards to its static CJMultiSlice
// (src/JMultiSliceLib.h:106, src/JMultiSliceLib.cpp).
#include "../../include/jms_b200.h"
#include "jms_host.h"
#include "jms_kernels.h"
#include "jms_pgr_host.h"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

using jms::JmsB200;

// Library contexts: context 0 is the default instance of the reference's flat
// interface; JMS_CreateContext adds more (each with its own grid, setup,
// device buffers and stream), and JMS_SelectContext picks the one the flat
// calls of the calling host thread act on.  The table holds shared pointers
// and every call works on its own copy, so a context that another thread
// destroys meanwhile is freed only when the last call using it returns.
namespace {
std::mutex g_ctx_mu;
std::vector<std::shared_ptr<JmsB200>> g_ctx;
thread_local int t_ctx = 0;

// with g_ctx_mu held
std::shared_ptr<JmsB200> ctx_get(int id)
{
	if (g_ctx.empty()) g_ctx.emplace_back(std::make_shared<JmsB200>());
	return (id >= 0 && id < (int)g_ctx.size()) ? g_ctx[id] : nullptr;
}
} // namespace

// the context of the calling thread (the default one if its context is gone)
static std::shared_ptr<JmsB200> J()
{
	std::lock_guard<std::mutex> lock(g_ctx_mu);
	std::shared_ptr<JmsB200> j = ctx_get(t_ctx);
	if (!j) {
		t_ctx = 0;
		j = ctx_get(0);
	}
	return j;
}

static jms::PgrGen& G()
{
	static std::unique_ptr<jms::PgrGen> inst(new jms::PgrGen());
	return *inst;
}

static int g_debug = 0;
static cudaStream_t g_pgr_stream = nullptr;   // generator stream (JMS_PgrSetStream); nullptr: the context's

extern "C" {

float GetJMSVersion(void) { return 0.46f; }
int SetJMSDebugLevel(int debuglevel) { int o = g_debug; g_debug = debuglevel; return o; }
void SeedRngEx(int rngseed) { J()->SeedRngEx(rngseed); }

float SetHighTension(float ht) { return J()->SetHighTension(ht); }
float GetHighTension(void) { return J()->GetHighTension(); }
float GetWaveLength(void) { return J()->GetWaveLength(); }
void SetSupercellSize(float* a0) { if (a0) J()->SetSupercellSize(a0[0], a0[1], a0[2]); }
void SetSupercellSizeABC(float a, float b, float c) { J()->SetSupercellSize(a, b, c); }
void SetSliceThickness(int islc, float fthickness) { J()->SetSliceThickness(islc, fthickness); }
void DiffractionDescan(int bActivate) { J()->DiffractionDescan(bActivate != 0); }
void SetPlasmonMC(int bActivate, float fq_e, float fq_c, float fmfp, unsigned int nexmax)
{ J()->SetPlasmonMC(bActivate != 0, fq_e, fq_c, fmfp, nexmax); }
void SetDiffractionDescanN(int whichcode, int ndescanx, int ndescany, int) { J()->SetDiffractionDescanN(whichcode, ndescanx, ndescany); }
void SetDiffractionDescan(int whichcode, float descanx, float descany, int) { J()->SetDiffractionDescan(whichcode, descanx, descany); }
void SetDiffractionDescanMRad(int whichcode, float descanx, float descany, int) { J()->SetDiffractionDescanMRad(whichcode, descanx, descany); }

void SetGridSize(int nx, int ny) { J()->SetGridSize(nx, ny); }
void GetGridSize(int* nx, int* ny) { int a = 0, b = 0; J()->GetGridSize(a, b); if (nx) *nx = a; if (ny) *ny = b; }
int GetDetetionSliceNum(void) { return J()->GetDetetionSliceNum(); }
int GetDetNum(void) { return J()->GetDetNum(); }
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
int GetCurrentGPU(void) { return J()->GetCurrentGPU(); }
int SetCurrentGPU(int idev) { return J()->SetCurrentGPU(idev); }
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
int GetUnscrambleHash(unsigned int* phash) { return J()->GetUnscrambleHash(phash); }
float GetImageAveragingWeight(int whichcode, int iThread) { return J()->GetImageAveragingWeight(whichcode, iThread); }
float GetWaveAveragingWeight(int whichcode, int iThread) { return J()->GetWaveAveragingWeight(whichcode, iThread); }

int PhaseGratingSetup(int whichcode, int nx, int ny, int nslc, int nvarmax, int* nslcvar)
{ return J()->PhaseGratingSetup(whichcode, nx, ny, nslc, nvarmax, nslcvar); }
int ObjectSliceSetup(int nobjslc, int* objslc) { return J()->ObjectSliceSetup(nobjslc, objslc); }
int PropagatorSetup(int whichcode, int npro, int* proidx) { return J()->PropagatorSetup(whichcode, npro, proidx); }
int DetectorSetup(int whichcode, int ndetper, int ndetint, int imagedet, int nthreads_CPU)
{ return J()->DetectorSetup(whichcode, ndetper, ndetint, imagedet, nthreads_CPU); }
int InitCore(int whichcode, int nCPUthreads) { return J()->InitCore(whichcode, nCPUthreads); }
int SetIncidentWave(int whichcode, float* wav) { return J()->SetIncidentWave(whichcode, wav, false); }
int SetIncidentWavePhaseplate(int whichcode, float* ppl, int bTranspose)
{ return J()->SetIncidentWavePhaseplate(whichcode, ppl, bTranspose != 0); }
int ZeroIncidentWavePhaseplate(int whichcode) { return J()->ZeroIncidentWavePhaseplate(whichcode); }
int SetSlicePhaseGratings(int whichcode, int islc, int nvar, float* pgr)
{ return J()->SetPhaseGratingData(whichcode, islc, nvar, pgr); }
int SetPropagatorData(int whichcode, int ipro, float* pro) { return J()->SetPropagatorData(whichcode, ipro, pro); }
int SetDetectorData(int whichcode, int idet, float* det, int msklen, int* msk)
{ return J()->SetDetectorData(whichcode, idet, det, msklen, msk); }
int SetGPUPgrLoading(int npgrload) { return J()->SetGPUPgrLoading(npgrload); }
int ResetImageAveraging(int whichcode, int iThread) { return J()->ResetImageAveraging(whichcode, iThread); }
int ResetWaveAveraging(int whichcode, int iThread) { return J()->ResetWaveAveraging(whichcode, iThread); }

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
	return J()->CalculateProbeWaveFourier(p, wav);
}
int SetIncomingWaveGPU(float* wav, int bTranspose) { return J()->SetIncomingWaveGPU(wav, bTranspose != 0); }
int SetIncomingWaveCPU(float*, int, int) { return 1; }
int CalculatePropagator(float fthick, float otx, float oty, float* pro, int ntype)
{ return J()->CalculatePropagator(fthick, otx, oty, pro, ntype); }
int CalculateRingDetector(float beta0, float beta1, float phi0, float phi1, float theta0x, float theta0y,
	const char* sdsprofile, float* det, int* msklen, int* msk, int kmom1)
{
	// the reference's flat interface passes theta0x twice (src/JMultiSliceLib.cpp:254);
	// here theta0y reaches the class as intended
	return J()->CalculateRingDetector(beta0, beta1, phi0, phi1, theta0x, theta0y, sdsprofile, det, msklen, msk, kmom1);
}
int OffsetIncomingWave(int whichcode, float dx, float dy, float dz, int iThread, int ibtx, int ibty)
{ return J()->OffsetIncomingWave(whichcode, dx, dy, dz, iThread, ibtx, ibty, true); }
int CPUMultislice(int, int, float, int) { return 1; }
int GPUMultislice(int islc0, int accmode, float weight) { return J()->GPUMultislice(islc0, accmode, weight); }
int GetResult(int whichcode, int whichresult, float* dst, int iThread)
{ return J()->GetResult(whichcode, whichresult, dst, iThread); }
int GetAvgResult(int whichcode, int whichresult, float* dst, float* wgt, int iThread)
{ return J()->GetAvgResult(whichcode, whichresult, dst, wgt, iThread); }
int ClearDetMem_h(int) { return 1; }
int ClearDetMem_d(void) { return J()->ClearDetMem_d(); }
int Cleanup(void) { return J()->Cleanup(); }
void FreeLibMem(void) {}

int JMS_SetStream(void* stream) { return J()->SetStream((cudaStream_t)stream); }
int JMS_ScanGPU(int npos, const float* pos, float dz, int npass, const int* varseq, float* out_int, float* out_bin,
	int bin)
{ return J()->ScanGPU(npos, pos, dz, npass, varseq, out_int, out_bin, bin); }
int JMS_ScanGPUDevice(int npos, const float* d_pos, float dz, int npass, const int* varseq, double* d_out_int,
	float* d_out_bin, int bin)
{ return J()->ScanGPUDevice(npos, d_pos, dz, npass, varseq, d_out_int, d_out_bin, bin); }
int JMS_SetScanBatch(int nwave) { return J()->SetScanBatch(nwave); }
int JMS_SetPassFusion(int on) { return J()->SetPassFusion(on); }

// Multi-fidelity frozen-phonon scan: the control-variate estimate
//   est = f(c0) + (npass - 1) / npass * (mean_{c1..} g - g(c0))
//       = f(c0) - (g(c0) - mean_{c0..} g)          (beta = 1)
// of the npass-configuration average of the full-grid context, from one
// full-grid pass (configuration c0) and npass passes of the coarse context.
// Both contexts run on their own streams (concurrently); the full context's
// stream waits for the coarse one before the combination.
int JMS_ScanMultiFidelityDevice(int ctx_full, int ctx_low, int npos, const float* d_pos, float dz, int npass,
	const int* varseq, double* d_out_int)
{
	std::shared_ptr<JmsB200> F, Lo;
	{
		std::lock_guard<std::mutex> lock(g_ctx_mu);
		F = ctx_get(ctx_full);
		Lo = ctx_get(ctx_low);
	}
	if (F == nullptr || Lo == nullptr || F == Lo) return 1;
	if (npos < 1 || npass < 1 || d_pos == nullptr || varseq == nullptr || d_out_int == nullptr) return 1;
	const int nd = F->GetDetetionSliceNum(), ndet = F->GetDetNum(), nobj = F->GetObjectSliceNum();
	if (nd != Lo->GetDetetionSliceNum() || ndet != Lo->GetDetNum() || nobj != Lo->GetObjectSliceNum() || nd < 1 ||
		ndet < 1)
		return 3;
	if (F->Stream() == nullptr || Lo->Stream() == nullptr) return 2;
	const size_t n = (size_t)npos * nd * ndet;
	// The coarse sums go to one half of the coarse context's control-variate
	// scratch; the combine that read this half two calls ago (on the full-grid
	// stream) must be done before the coarse stream clears it.
	cudaEvent_t done = nullptr;
	double* g = Lo->CvScratch(n, &done);
	if (g == nullptr || done == nullptr) return 4;
	double *g1 = g, *gm = g + n;
	cudaStream_t sf = F->Stream(), sl = Lo->Stream();
	if (cudaStreamWaitEvent(sl, done, 0) != cudaSuccess) return 5;
	if (cudaMemsetAsync(d_out_int, 0, sizeof(double) * n, sf) != cudaSuccess) return 5;
	if (cudaMemsetAsync(g, 0, sizeof(double) * 2 * n, sl) != cudaSuccess) return 5;
	int e = F->ScanGPUDevice(npos, d_pos, dz, 1, varseq, d_out_int, nullptr, 0);
	if (e) return e;
	e = Lo->ScanGPUDevice(npos, d_pos, dz, 1, varseq, g1, nullptr, 0);
	if (e) return e;
	if (npass > 1) {
		e = Lo->ScanGPUDevice(npos, d_pos, dz, npass - 1, varseq + nobj, gm, nullptr, 0);
		if (e) return e;
		cudaEvent_t ev;
		if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) return 5;
		cudaEventRecord(ev, sl);
		cudaStreamWaitEvent(sf, ev, 0);
		cudaEventDestroy(ev);
		if (jms::launch_cv_combine(d_out_int, g1, gm, (long long)n, (double)(npass - 1) / (double)npass, sf) !=
			cudaSuccess)
			return 5;
		if (cudaEventRecord(done, sf) != cudaSuccess) return 5;   // this half is free again after the combine
	}
	return 0;
}

int JMS_ScanMultiFidelity(int ctx_full, int ctx_low, int npos, const float* pos, float dz, int npass,
	const int* varseq, float* out_int)
{
	if (npos < 1 || pos == nullptr || out_int == nullptr) return 1;
	std::shared_ptr<JmsB200> F;
	{
		std::lock_guard<std::mutex> lock(g_ctx_mu);
		F = ctx_get(ctx_full);
	}
	if (F == nullptr || F->Stream() == nullptr) return 1;
	const size_t n = (size_t)npos * std::max(1, F->GetDetetionSliceNum()) * std::max(1, F->GetDetNum());
	// device copies of the positions and the estimate, in the full context's scratch
	double* d = F->Scratch(n + (size_t)npos);
	if (d == nullptr) return 4;
	double* d_out = d;
	float* d_pos = reinterpret_cast<float*>(d + n);
	cudaStream_t sf = F->Stream();
	if (cudaMemcpyAsync(d_pos, pos, sizeof(float) * 2 * (size_t)npos, cudaMemcpyHostToDevice, sf) != cudaSuccess)
		return 5;
	if (cudaStreamSynchronize(sf) != cudaSuccess) return 5;    // the coarse context reads d_pos on its own stream
	int e = JMS_ScanMultiFidelityDevice(ctx_full, ctx_low, npos, d_pos, dz, npass, varseq, d_out);
	if (e) return e;
	std::vector<double> h(n);
	if (cudaMemcpyAsync(h.data(), d_out, sizeof(double) * n, cudaMemcpyDeviceToHost, sf) != cudaSuccess) return 5;
	if (cudaStreamSynchronize(sf) != cudaSuccess) return 5;
	for (size_t i = 0; i < n; i++) out_int[i] = (float)h[i];
	return 0;
}
long long JMS_KernelLaunches(void) { return J()->KernelLaunches(); }
void JMS_SetPassTiming(int on) { J()->SetPassTiming(on); }
int JMS_PassTiming(double* ms_col, long long* n_col, double* ms_row, long long* n_row)
{ return J()->PassTiming(ms_col, n_col, ms_row, n_row); }
int JMS_ReadoutDetectorsNoAlloc(const float* d_wav, int nwave, double* d_out, void* stream)
{ return J()->ReadoutDetectorsNoAlloc(d_wav, nwave, d_out, (cudaStream_t)stream); }
int JMS_Autotune(int nwave, int reps, float* ms_row, float* ms_col, int* irow, int* icol)
{ return J()->Autotune(nwave, reps, ms_row, ms_col, irow, icol); }
int JMS_SelectPlans(int irow, int icol) { return J()->SelectPlans(irow, icol); }
int JMS_PlanCount(int n) { return jms::plan_count(n); }
int JMS_PlanName(int axis, char* name, int len)
{
	if (!name || len < 1) return 1;
	std::strncpy(name, J()->PlanName(axis), (size_t)len - 1);
	name[len - 1] = 0;
	return 0;
}
int JMS_GridSupported(int nx, int ny) { return (jms::pass_supported(nx) && jms::pass_supported(ny)) ? 1 : 0; }
int JMS_SetPrecision(int mode) { return J()->SetPrecision(mode); }
int JMS_GetPrecision(void) { return J()->GetPrecision(); }
int JMS_TcStatus(void) { return J()->TcStatus(); }
long long JMS_TcLaunches(void) { return J()->TcLaunches(); }

int JMS_ReadoutDetAvg(int whichcode, int whichresult, float* dst, float* weight)
{ return J()->ReadoutDetAvg(whichcode, whichresult, dst, weight, 0); }

int JMS_CreateContext(void)
{
	std::lock_guard<std::mutex> lock(g_ctx_mu);
	ctx_get(0);
	for (size_t i = 1; i < g_ctx.size(); i++)
		if (!g_ctx[i]) { g_ctx[i] = std::make_shared<JmsB200>(); return (int)i; }
	g_ctx.emplace_back(std::make_shared<JmsB200>());
	return (int)g_ctx.size() - 1;
}

int JMS_SelectContext(int id)
{
	std::lock_guard<std::mutex> lock(g_ctx_mu);
	if (!ctx_get(id)) return -1;
	const int old = t_ctx;
	t_ctx = id;
	return old;
}

int JMS_DestroyContext(int id)
{
	std::shared_ptr<JmsB200> victim;
	{
		std::lock_guard<std::mutex> lock(g_ctx_mu);
		if (id <= 0 || !ctx_get(id)) return 1;
		victim = std::move(g_ctx[id]);
		if (t_ctx == id) t_ctx = 0;
	}
	return 0;   // freed here, outside the lock, unless a call on another thread still holds it
}

// ---- CUDA graphs over contexts -------------------------------------------
namespace {
struct GraphRec {
	cudaGraph_t graph = nullptr;
	cudaGraphExec_t exec = nullptr;
};
std::mutex g_graph_mu;
std::vector<std::unique_ptr<GraphRec>> g_graphs;
cudaStream_t g_origin = nullptr;
std::vector<cudaStream_t> g_cap_streams;
bool g_capturing = false;
} // namespace

int JMS_GraphBegin(int nctx, const int* ctx)
{
	std::lock_guard<std::mutex> lock(g_graph_mu);
	if (g_capturing || nctx < 1 || ctx == nullptr) return 1;
	std::vector<cudaStream_t> streams;
	{
		std::lock_guard<std::mutex> lk(g_ctx_mu);
		for (int i = 0; i < nctx; i++) {
			std::shared_ptr<JmsB200> j = ctx_get(ctx[i]);
			if (!j) return 1;
			if (j->Stream() == nullptr) return 2;   // the context needs its stream (InitCore)
			for (cudaStream_t q : streams)
				if (q == j->Stream()) return 1;
			streams.push_back(j->Stream());
		}
	}
	if (g_origin == nullptr && cudaStreamCreateWithFlags(&g_origin, cudaStreamNonBlocking) != cudaSuccess) return 3;
	if (cudaStreamBeginCapture(g_origin, cudaStreamCaptureModeRelaxed) != cudaSuccess) return 3;
	cudaEvent_t fork;
	cudaEventCreateWithFlags(&fork, cudaEventDisableTiming);
	cudaEventRecord(fork, g_origin);
	for (cudaStream_t q : streams) cudaStreamWaitEvent(q, fork, 0);
	cudaEventDestroy(fork);
	g_cap_streams = streams;
	g_capturing = true;
	return 0;
}

int JMS_GraphEnd(void)
{
	std::lock_guard<std::mutex> lock(g_graph_mu);
	if (!g_capturing) return -1;
	g_capturing = false;
	for (cudaStream_t q : g_cap_streams) {
		cudaEvent_t join;
		cudaEventCreateWithFlags(&join, cudaEventDisableTiming);
		cudaEventRecord(join, q);
		cudaStreamWaitEvent(g_origin, join, 0);
		cudaEventDestroy(join);
	}
	g_cap_streams.clear();
	std::unique_ptr<GraphRec> r(new GraphRec());
	if (cudaStreamEndCapture(g_origin, &r->graph) != cudaSuccess || r->graph == nullptr) {
		cudaGetLastError();
		return -2;
	}
	if (cudaGraphInstantiate(&r->exec, r->graph, 0) != cudaSuccess) {
		cudaGraphDestroy(r->graph);
		cudaGetLastError();
		return -3;
	}
	for (size_t i = 0; i < g_graphs.size(); i++)
		if (!g_graphs[i]) { g_graphs[i] = std::move(r); return (int)i + 1; }
	g_graphs.push_back(std::move(r));
	return (int)g_graphs.size();
}

int JMS_GraphLaunch(int handle, void* stream, int wait)
{
	cudaGraphExec_t x = nullptr;
	{
		std::lock_guard<std::mutex> lock(g_graph_mu);
		if (handle < 1 || handle > (int)g_graphs.size() || !g_graphs[handle - 1]) return 1;
		x = g_graphs[handle - 1]->exec;
	}
	cudaStream_t s = stream ? (cudaStream_t)stream : g_origin;
	if (cudaGraphLaunch(x, s) != cudaSuccess) return 2;
	if (wait && cudaStreamSynchronize(s) != cudaSuccess) return 3;
	return 0;
}

int JMS_GraphDestroy(int handle)
{
	std::lock_guard<std::mutex> lock(g_graph_mu);
	if (handle < 1 || handle > (int)g_graphs.size() || !g_graphs[handle - 1]) return 1;
	GraphRec* r = g_graphs[handle - 1].get();
	cudaGraphExecDestroy(r->exec);
	cudaGraphDestroy(r->graph);
	g_graphs[handle - 1].reset();
	return 0;
}

int JMS_SliLoadSlice(const char* path, int islc)
{
	JMSSliHeader h;
	int e = JMS_SliReadHeader(path, &h);
	if (e) return e;
	int npgx = 0, npgy = 0;
	if (J()->GratingSlot(islc, 0, 1, &npgx, &npgy) == nullptr) return 1;
	if (h.nx != npgx || h.ny != npgy) return 7;
	std::vector<float> buf((size_t)2 * h.nx * h.ny * h.nvar);
	if ((e = JMS_SliReadData(path, buf.data()))) return e;
	return J()->SetPhaseGratingData(jms::CODE_GPU, islc, h.nvar, buf.data());
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
int JMS_PgrSetStream(void* stream)
{
	g_pgr_stream = (cudaStream_t)stream;
	return 0;
}
int JMS_PgrCalculate(int natom, const float* atoms, float cz, int ngr, unsigned long long seed, int islc, int ivar0,
	float* pgr)
{
	float2* dst = nullptr;
	if (islc >= 0) {
		int npgx = 0, npgy = 0;
		dst = J()->GratingSlot(islc, ivar0, ngr, &npgx, &npgy);
		if (dst == nullptr || npgx != G().nx() || npgy != G().ny()) return 9;
	}
	cudaStream_t s = g_pgr_stream ? g_pgr_stream : J()->Stream();
	G().SetStream(s);
	int e = G().Calculate(natom, atoms, cz, ngr, seed, dst, pgr);
	// before InitCore the context has no stream of its own yet, and the one it
	// creates does not wait for the legacy stream: finish the gratings here
	if (e == 0 && dst != nullptr && s == nullptr && cudaStreamSynchronize(nullptr) != cudaSuccess) e = 7;
	return e;
}

} // extern "C"
