// class_case.cpp -- a caller of the C++ class interface (include/JMultiSlice.h),
// built and run by tests/test_class_interface.py.  It uses the library the way
// the reference's benchmark driver does (test/JMSBench1/multislice.cpp:251-688:
// a CJMultiSlice object, its setup chain, then OffsetIncomingWave /
// GPUMultislice / GetResult per run), with the default arguments of the
// reference's header.  Inputs and outputs are raw little-endian arrays in a
// directory, named as below; the test writes the inputs from its golden
// vectors and compares the outputs.
//
//   class_case gen  DIR   generators only (no GPU): probes, propagators and
//                          ring detectors of the reference's generator cases
//   class_case run  DIR   one golden multislice case on the GPU, plus the
//                          frozen-phonon variant draws of two seeds
#include "JMultiSlice.h"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

namespace {

template <class T>
std::vector<T> load(const std::string& dir, const std::string& name)
{
	std::ifstream f(dir + "/" + name, std::ios::binary | std::ios::ate);
	if (!f) {
		std::fprintf(stderr, "missing input %s\n", name.c_str());
		std::exit(3);
	}
	const size_t n = (size_t)f.tellg() / sizeof(T);
	std::vector<T> v(n);
	f.seekg(0);
	f.read((char*)v.data(), n * sizeof(T));
	return v;
}

template <class T>
void save(const std::string& dir, const std::string& name, const T* p, size_t n)
{
	std::ofstream f(dir + "/" + name, std::ios::binary);
	f.write((const char*)p, n * sizeof(T));
}

// exposes the protected variant draw, as a subclass of the reference class can
class DrawingJMS : public CJMultiSlice {
public:
	using CJMultiSlice::GetRandomVariantSequence;
};

int check(int e, const char* what)
{
	if (e != 0) std::fprintf(stderr, "%s returned %d\n", what, e);
	return e;
}

// generators: gen.f32 = ht, nx, ny, a, b, c, then per probe 8 parameters +
// 48 aberration coefficients (nprobe from gen_n.i32[0]), then per detector 7
// values (beta0, beta1, phi0, phi1, theta0x, theta0y, kmom) (ndet = gen_n.i32[1])
int run_gen(const std::string& dir)
{
	const std::vector<float> g = load<float>(dir, "gen.f32");
	const std::vector<int> n = load<int>(dir, "gen_n.i32");
	CJMultiSlice jms;
	jms.SetHighTension(g[0]);
	const int nx = (int)g[1], ny = (int)g[2];
	jms.SetGridSize(nx, ny);
	jms.SetSupercellSize(g[3], g[4], g[5]);
	size_t k = 6;
	std::vector<fcmplx> wav((size_t)nx * ny);
	for (int ip = 0; ip < n[0]; ip++) {
		CJProbeParams prm;
		prm.m_alpha = g[k + 0];
		prm.m_alpha_rs = g[k + 1];
		prm.m_alpha_x0 = g[k + 2];
		prm.m_alpha_y0 = g[k + 3];
		prm.m_alpha_asym = g[k + 4];
		prm.m_alpha_adir = g[k + 5];
		prm.m_btx = g[k + 6];
		prm.m_bty = g[k + 7];
		for (int i = 0; i < 2 * prm.GetAberrationNum(); i++) prm.m_abrr_coeff[i] = g[k + 8 + i];
		k += 8 + 48;
		CJProbeParams copy(prm);   // the copy carries every field
		if (!(copy == prm)) return 10;
		if (check(jms.CalculateProbeWaveFourier(&copy, wav.data()), "CalculateProbeWaveFourier")) return 11;
		save(dir, "probe" + std::to_string(ip) + ".c64", wav.data(), wav.size());
	}
	std::vector<fcmplx> pro((size_t)nx * ny);
	std::vector<float> det((size_t)nx * ny);
	std::vector<int> msk((size_t)nx * ny);
	for (int nt = 0; nt < 2; nt++) {
		if (check(jms.CalculatePropagator(0.19525f, 0.f, 0.f, pro.data(), nt), "CalculatePropagator")) return 12;
		save(dir, "pro_t" + std::to_string(nt) + ".c64", pro.data(), pro.size());
		if (check(jms.CalculatePropagator(0.25f, 0.5f, -0.3f, pro.data(), nt), "CalculatePropagator")) return 12;
		save(dir, "pro_t" + std::to_string(nt) + "_tilt.c64", pro.data(), pro.size());
		for (int id = 0; id < n[1]; id++) {
			const float* d = &g[k + 7 * id];
			int msklen = 0;
			if (check(jms.CalculateRingDetector(d[0], d[1], d[2], d[3], d[4], d[5], "", det.data(), msklen,
				msk.data(), (int)d[6]), "CalculateRingDetector")) return 13;
			const std::string s = std::to_string(nt) + "_" + std::to_string(id);
			save(dir, "det_t" + s + ".f32", det.data(), det.size());
			save(dir, "msk_t" + s + ".i32", msk.data(), (size_t)msklen);
		}
	}
	// the probe defaults of the reference class, and its wavelength formula
	CJProbeParams d;
	float dv[4] = {d.m_wl, d.m_alpha, d.m_alpha_rs, d.SetProbeEkV(300.f)};
	save(dir, "probe_defaults.f32", dv, 4);
	return 0;
}

// one multislice case: cfg.i32 = nx, ny, npgx, npgy, ndetper, imagedet, seed,
// islc0, ndet, nslc, npro, nobj, nrun; cell.f32 = a, b, kv; nvar.i32,
// objslc.i32, proidx.i32; pgr<s>.c64, pro<i>.c64, det<i>.f32, msk<i>.i32,
// probe.c64; cppl.f32 (optional constant phase plate); runs.f32 = nrun x (dx, dy, dz, ibtx, ibty, accmode, weight);
// draws_nvar.i32 / draws_obj.i32: variants per structure slice and object
// slices of the variant-draw check
int run_case(const std::string& dir)
{
	const std::vector<int> cfg = load<int>(dir, "cfg.i32");
	const std::vector<float> cell = load<float>(dir, "cell.f32");
	std::vector<int> nvar = load<int>(dir, "nvar.i32");
	std::vector<int> objslc = load<int>(dir, "objslc.i32");
	std::vector<int> proidx = load<int>(dir, "proidx.i32");
	const std::vector<float> runs = load<float>(dir, "runs.f32");
	const int nx = cfg[0], ny = cfg[1], npgx = cfg[2], npgy = cfg[3], ndetper = cfg[4], imagedet = cfg[5];
	const int seed = cfg[6], islc0 = cfg[7], ndet = cfg[8], nslc = cfg[9], npro = cfg[10], nobj = cfg[11];
	const int nrun = cfg[12];
	const int gpu = _JMS_CODE_GPU;

	CJMultiSlice* pjms = new CJMultiSlice();
	pjms->SetHighTension(cell[2]);
	pjms->SetGridSize(nx, ny);
	pjms->SetSupercellSize(cell[0], cell[1], 0.4f);
	pjms->SetGPUPgrLoading();
	if (pjms->GetGPUNum() < 1) return 20;
	int nvarmax = 0;
	for (int v : nvar) nvarmax = std::max(nvarmax, v);
	if (check(pjms->PhaseGratingSetup(gpu, npgx, npgy, nslc, nvarmax, nvar.data()), "PhaseGratingSetup")) return 21;
	if (check(pjms->ObjectSliceSetup(nobj, objslc.data()), "ObjectSliceSetup")) return 22;
	if (check(pjms->PropagatorSetup(gpu, npro, proidx.data()), "PropagatorSetup")) return 23;
	if (check(pjms->DetectorSetup(gpu, ndetper, ndet, imagedet), "DetectorSetup")) return 24;
	for (int s = 0; s < nslc; s++) {
		std::vector<fcmplx> pgr = load<fcmplx>(dir, "pgr" + std::to_string(s) + ".c64");
		if (check(pjms->SetPhaseGratingData(gpu, s, nvar[s], pgr.data()), "SetPhaseGratingData")) return 25;
	}
	for (int i = 0; i < npro; i++) {
		std::vector<fcmplx> pro = load<fcmplx>(dir, "pro" + std::to_string(i) + ".c64");
		if (check(pjms->SetPropagatorData(gpu, i, pro.data()), "SetPropagatorData")) return 26;
	}
	for (int i = 0; i < ndet; i++) {
		std::vector<float> det = load<float>(dir, "det" + std::to_string(i) + ".f32");
		std::vector<int> msk = load<int>(dir, "msk" + std::to_string(i) + ".i32");
		const int e = msk.empty() ? pjms->SetDetectorData(gpu, i, det.data())
		                          : pjms->SetDetectorData(gpu, i, det.data(), (int)msk.size(), msk.data());
		if (check(e, "SetDetectorData")) return 27;
	}
	if (check(pjms->InitCore(gpu), "InitCore")) return 28;
	std::vector<fcmplx> probe = load<fcmplx>(dir, "probe.c64");
	if (check(pjms->SetIncidentWave(gpu, probe.data()), "SetIncidentWave")) return 29;
	if (std::ifstream(dir + "/cppl.f32").good()) {   // constant phase plate of the case, if any
		std::vector<float> cppl = load<float>(dir, "cppl.f32");
		if (check(pjms->SetIncidentWavePhaseplate(gpu, cppl.data()), "SetIncidentWavePhaseplate")) return 29;
	}
	pjms->SeedRngEx(seed);
	for (int r = 0; r < nrun; r++) {
		const float* q = &runs[(size_t)7 * r];
		if (check(pjms->OffsetIncomingWave(gpu, q[0], q[1], q[2], 0, (int)q[3], (int)q[4]), "OffsetIncomingWave"))
			return 30;
		if (check(pjms->GPUMultislice(islc0, (int)q[5], q[6]), "GPUMultislice")) return 31;
	}
	const int nd = pjms->GetDetetionSliceNum();
	const size_t N = (size_t)nx * ny, L = N * nd;
	int dims[2] = {nd, pjms->GetDetNum()};
	save(dir, "out_dims.i32", dims, 2);
	if (imagedet & _JMS_DETECT_INTEGRATED) {
		std::vector<float> v((size_t)nd * ndet);
		if (check(pjms->GetResult(gpu, _JMS_DETECT_INTEGRATED, v.data()), "GetResult")) return 32;
		save(dir, "out_det_int.f32", v.data(), v.size());
	}
	const struct { int flag; const char* name; int cplx; } ch[] = {
		{_JMS_DETECT_IMAGE, "out_img.f32", 0}, {_JMS_DETECT_DIFFRACTION, "out_dif.f32", 0},
		{_JMS_DETECT_WAVEREAL, "out_wfr.c64", 1}, {_JMS_DETECT_WAVEFOURIER, "out_wff.c64", 1}};
	for (const auto& c : ch) {
		if (!(imagedet & c.flag)) continue;
		std::vector<float> v(L * (c.cplx ? 2 : 1));
		if (check(pjms->GetResult(gpu, c.flag, v.data()), "GetResult")) return 33;
		save(dir, c.name, v.data(), v.size());
	}
	std::vector<unsigned int> hash(N);
	if (check(pjms->GetUnscrambleHash(hash.data()), "GetUnscrambleHash")) return 34;
	save(dir, "out_unscramble.u32", hash.data(), N);
	delete pjms;

	// frozen-phonon variant draws through a subclass (seeds 11 and 12, three
	// draws each), with a CPU-code setup refused and a GPU-code one accepted
	std::vector<int> dn = load<int>(dir, "draws_nvar.i32");
	std::vector<int> dobj = load<int>(dir, "draws_obj.i32");
	std::vector<int> out;
	for (int sd : {11, 12}) {
		DrawingJMS d;
		d.SetHighTension(300.f);
		d.SetGridSize(8, 8);
		d.SetSupercellSize(1.f, 1.f, 1.f);
		int mx = 0;
		for (int v : dn) mx = std::max(mx, v);
		if (d.PhaseGratingSetup(_JMS_CODE_CPU, 8, 8, (int)dn.size(), mx, dn.data()) != 1) return 40;
		if (check(d.PhaseGratingSetup(gpu, 8, 8, (int)dn.size(), mx, dn.data()), "PhaseGratingSetup")) return 41;
		if (check(d.ObjectSliceSetup((int)dobj.size(), dobj.data()), "ObjectSliceSetup")) return 42;
		CRng own(sd);                 // a caller's generator, handed to the object
		d.SetRng(&own);
		if (d.GetRng() != &own) return 43;
		std::vector<int> seq(dobj.size());
		for (int k = 0; k < 3; k++) {
			if (check(d.GetRandomVariantSequence(seq.data()), "GetRandomVariantSequence")) return 44;
			out.insert(out.end(), seq.begin(), seq.end());
		}
		d.SetRng(NULL);
	}
	save(dir, "out_draws.i32", out.data(), out.size());
	return 0;
}

} // namespace

int main(int argc, char** argv)
{
	if (argc != 3) {
		std::fprintf(stderr, "usage: class_case gen|run DIR\n");
		return 2;
	}
	const std::string mode = argv[1], dir = argv[2];
	if (mode == "gen") return run_gen(dir);
	if (mode == "run") return run_case(dir);
	return 2;
}
