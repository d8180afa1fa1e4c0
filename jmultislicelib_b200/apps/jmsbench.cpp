// jmsbench.cpp -- STEM driver compatible with the reference's bench program
// (test/JMSBench1) for slice-file input, running the scan through the C ABI
// of libjms_b200 (include/jms_b200.h) on one GPU.
//
//   jmsbench <control file> [/o <output prefix>]
//
// Control-file commands (test/JMSBench1/input_command.txt): a keyword line,
// then its data line.  Supported: set_gpu_id, set_cpu_num (ignored),
// set_sample_input_form (2 = slice files), set_slc_num, set_slc_file_name,
// set_sample_thickness_max, set_sample_thickness_step, set_sample_tilt,
// set_probe_ekv, set_probe_convergence, set_probe_aberration,
// set_det_annular, set_scan_sampling, set_scan_frame_size,
// set_scan_frame_rot, set_scan_beam_pos, set_num_repeat, set_output_file.
// Other commands stop the run with a message.
//
// Semantics followed from the reference bench:
//   slice files <prefix>_001.sli, _002.sli, ... (prm_sample.cpp:466-486),
//   object slice i = structure slice i % nslc (prm_sample.cpp:297-301),
//   readout every <step> slices plus entrance and exit planes
//   (prm_sample.cpp:284-315; the period form of DetectorSetup),
//   planar propagators with the object tilt in mrad (prm_slice.cpp:495-516),
//   probe edge smoothness 0.03 by default (prm_probe.cpp:37, 477-500),
//   scan pixel (ix, iy) at offset + R(rot) (step_x ix, step_y iy)
//   (multislice.cpp:876-877), repeats averaged (multislice.cpp:908-909),
//   one file per detector <output>_<name>.bin holding float
//   [plane][scan y][scan x] (prm_main.cpp:599-602, prm_result.cpp:192-290).
#include "../../include/jms_b200.h"

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

namespace {

struct Annular {
	float b0 = 0.f, b1 = 0.f, p0 = 0.f, p1 = 0.f;
	std::string name;
};

std::string unquote(std::string s)
{
	while (!s.empty() && (s.back() == '\r' || s.back() == ' ' || s.back() == '\t')) s.pop_back();
	size_t a = s.find_first_not_of(" \t");
	s = (a == std::string::npos) ? std::string() : s.substr(a);
	if (s.size() >= 2 && (s.front() == '\'' || s.front() == '"') && s.back() == s.front()) s = s.substr(1, s.size() - 2);
	return s;
}

std::vector<std::string> words(const std::string& line)
{
	std::istringstream is(line);
	std::vector<std::string> w;
	std::string t;
	while (is >> t) w.push_back(t);
	return w;
}

int fail(const char* msg, const std::string& what = "")
{
	std::fprintf(stderr, "Error (jmsbench): %s%s\n", msg, what.c_str());
	return 1;
}

} // namespace

int main(int argc, char** argv)
{
	if (argc < 2) {
		std::fprintf(stderr, "usage: jmsbench <control file> [/o <output prefix>]\n");
		return 2;
	}
	std::string out_file = "output";
	for (int i = 2; i + 1 < argc; i++)
		if (std::strcmp(argv[i], "/o") == 0 || std::strcmp(argv[i], "-o") == 0) out_file = argv[i + 1];
	std::ifstream in(argv[1]);
	if (!in) return fail("cannot open control file ", argv[1]);
	std::multimap<std::string, std::string> cmd;
	std::string line, key;
	while (std::getline(in, line)) {
		std::string t = unquote(line);
		if (t.rfind("set_", 0) == 0 && t.find(' ') == std::string::npos) {
			key = t;
			// commands without a data line
			if (key == "set_det_dif" || key == "set_det_padif" || key == "set_det_img" || key == "set_det_paimg" ||
				key == "set_det_separate_tds") cmd.emplace(key, "");
		}
		else if (!key.empty()) {
			cmd.emplace(key, line);
			key.clear();
		}
	}
	static const char* known[] = {"set_gpu_id", "set_cpu_num", "set_sample_input_form", "set_slc_num",
		"set_slc_file_name", "set_sample_thickness_max", "set_sample_thickness_step", "set_sample_tilt",
		"set_probe_ekv", "set_probe_convergence", "set_probe_aberration", "set_det_annular", "set_scan_sampling",
		"set_scan_frame_size", "set_scan_frame_rot", "set_scan_beam_pos", "set_num_repeat", "set_output_file"};
	for (auto& kv : cmd) {
		bool ok = false;
		for (const char* k : known) ok = ok || kv.first == k;
		if (!ok) return fail("unsupported control command ", kv.first);
	}
	auto get = [&](const char* k) -> std::string {
		auto it = cmd.find(k);
		return it == cmd.end() ? std::string() : it->second;
	};
	if (!get("set_output_file").empty() && out_file == "output") out_file = unquote(get("set_output_file"));
	if (!get("set_sample_input_form").empty() && std::stoi(get("set_sample_input_form")) != 2)
		return fail("only slice-file input (set_sample_input_form 2) is supported");
	const std::string prefix = unquote(get("set_slc_file_name"));
	if (prefix.empty()) return fail("missing set_slc_file_name");
	if (!get("set_gpu_id").empty() && SetCurrentGPU(std::stoi(get("set_gpu_id"))) != 0) return fail("cannot select the GPU");

	// slice files
	std::vector<JMSSliHeader> hdr;
	std::vector<std::string> files;
	for (int i = 1; i < 1000; i++) {
		char name[64];
		std::snprintf(name, sizeof(name), "_%03d.sli", i);
		JMSSliHeader h;
		if (JMS_SliReadHeader((prefix + name).c_str(), &h) != 0) break;
		hdr.push_back(h);
		files.push_back(prefix + name);
	}
	const int nslc = (int)hdr.size();
	if (nslc == 0) return fail("no slice files found with prefix ", prefix);
	const int nx = hdr[0].nx, ny = hdr[0].ny;
	int nvarmax = 1;
	std::vector<int> nvar(nslc);
	float cz = 0.f;
	for (int i = 0; i < nslc; i++) {
		if (hdr[i].nx != nx || hdr[i].ny != ny) return fail("slice files of different grid sizes");
		nvar[i] = hdr[i].nvar;
		nvarmax = nvar[i] > nvarmax ? nvar[i] : nvarmax;
		cz += hdr[i].thickness;
	}
	const int nobj = get("set_sample_thickness_max").empty() ? nslc : std::stoi(get("set_sample_thickness_max"));
	const int step = get("set_sample_thickness_step").empty() ? 0 : std::stoi(get("set_sample_thickness_step"));
	float tilt_x = 0.f, tilt_y = 0.f;
	if (!get("set_sample_tilt").empty()) {
		auto w = words(get("set_sample_tilt"));
		if (w.size() >= 2) { tilt_x = std::stof(w[0]); tilt_y = std::stof(w[1]); }
	}
	const float ekv = get("set_probe_ekv").empty() ? hdr[0].ekv : std::stof(get("set_probe_ekv"));

	// physics, grid and setup chain
	SetGridSize(nx, ny);
	SetHighTension(ekv);
	SetSupercellSizeABC(hdr[0].sx, hdr[0].sy, cz);
	if (PhaseGratingSetup(JMS_CODE_GPU, nx, ny, nslc, nvarmax, nvar.data())) return fail("PhaseGratingSetup failed");
	std::vector<int> objslc(nobj), proidx(nslc);
	for (int i = 0; i < nobj; i++) objslc[i] = i % nslc;
	for (int i = 0; i < nslc; i++) proidx[i] = i;
	if (ObjectSliceSetup(nobj, objslc.data())) return fail("ObjectSliceSetup failed");
	if (PropagatorSetup(JMS_CODE_GPU, nslc, proidx.data())) return fail("PropagatorSetup failed");
	std::vector<Annular> ann;
	for (auto it = cmd.lower_bound("set_det_annular"); it != cmd.upper_bound("set_det_annular"); ++it) {
		auto w = words(it->second);
		if (w.size() < 5) return fail("set_det_annular needs: inner outer azimuth-begin azimuth-end name");
		Annular a;
		a.b0 = std::stof(w[0]); a.b1 = std::stof(w[1]); a.p0 = std::stof(w[2]); a.p1 = std::stof(w[3]);
		a.name = unquote(w[4]);
		ann.push_back(a);
	}
	if (ann.empty()) return fail("no annular detector (set_det_annular)");
	if (DetectorSetup(JMS_CODE_GPU, step, (int)ann.size(), JMS_DETECT_INTEGRATED, 0)) return fail("DetectorSetup failed");
	for (int i = 0; i < nslc; i++) {
		if (JMS_SliLoadSlice(files[i].c_str(), i)) return fail("cannot load ", files[i]);
		SetSliceThickness(i, hdr[i].thickness);
	}
	const size_t N = (size_t)nx * ny;
	std::vector<float> buf(2 * N);
	const float ttf = (float)(180.0 / 3.141592653589793) * 0.001f;   // mrad -> deg
	for (int i = 0; i < nslc; i++) {
		if (CalculatePropagator(hdr[i].thickness, ttf * tilt_x, ttf * tilt_y, buf.data(), 0)) return fail("CalculatePropagator failed");
		if (SetPropagatorData(JMS_CODE_GPU, i, buf.data())) return fail("SetPropagatorData failed");
	}
	std::vector<float> det(N);
	std::vector<int> msk(N);
	for (size_t i = 0; i < ann.size(); i++) {
		int msklen = 0;
		if (CalculateRingDetector(ann[i].b0, ann[i].b1, ann[i].p0, ann[i].p1, 0.f, 0.f, "", det.data(), &msklen,
			msk.data(), 0)) return fail("CalculateRingDetector failed");
		if (SetDetectorData(JMS_CODE_GPU, (int)i, det.data(), msklen, msk.data())) return fail("SetDetectorData failed");
	}
	if (InitCore(JMS_CODE_GPU, 0)) return fail("InitCore failed");

	// probe
	std::vector<float> abrr(48, 0.f);
	for (auto it = cmd.lower_bound("set_probe_aberration"); it != cmd.upper_bound("set_probe_aberration"); ++it) {
		auto w = words(it->second);
		if (w.size() < 3) return fail("set_probe_aberration needs: index x y");
		const int k = std::stoi(w[0]) - 1;
		if (k < 0 || k >= 24) return fail("aberration index out of range");
		abrr[2 * k] = std::stof(w[1]);
		abrr[2 * k + 1] = std::stof(w[2]);
	}
	JMSProbeParams prm;
	std::memset(&prm, 0, sizeof(prm));
	prm.m_alpha_rs = 0.03f;
	auto cw = words(get("set_probe_convergence"));
	if (cw.empty()) return fail("missing set_probe_convergence");
	prm.m_alpha = std::stof(cw[0]);
	if (cw.size() > 1) prm.m_alpha_rs = std::stof(cw[1]);
	if (cw.size() > 2) prm.m_alpha_asym = std::stof(cw[2]);
	if (cw.size() > 3) prm.m_alpha_adir = std::stof(cw[3]);
	prm.m_wl = GetWaveLength();
	prm.m_abrr_coeff = abrr.data();
	if (CalculateProbeWaveFourier(&prm, buf.data())) return fail("CalculateProbeWaveFourier failed");
	if (SetIncidentWave(JMS_CODE_GPU, buf.data())) return fail("SetIncidentWave failed");

	// scan positions
	int snx = 1, sny = 1;
	float fsx = 0.f, fsy = 0.f, rot = 0.f, offx = 0.f, offy = 0.f;
	if (!get("set_scan_sampling").empty()) { auto w = words(get("set_scan_sampling")); snx = std::stoi(w.at(0)); sny = std::stoi(w.at(1)); }
	if (!get("set_scan_frame_size").empty()) { auto w = words(get("set_scan_frame_size")); fsx = std::stof(w.at(0)); fsy = std::stof(w.at(1)); }
	if (!get("set_scan_frame_rot").empty()) rot = std::stof(get("set_scan_frame_rot")) * 3.14159265f / 180.f;
	if (!get("set_scan_beam_pos").empty()) { auto w = words(get("set_scan_beam_pos")); offx = std::stof(w.at(0)); offy = std::stof(w.at(1)); }
	const int nrep = get("set_num_repeat").empty() ? 1 : std::stoi(get("set_num_repeat"));
	if (snx < 1 || sny < 1 || nrep < 1) return fail("invalid scan sampling or repeats");
	const float stx = fsx / (float)snx, sty = fsy / (float)sny, cr = std::cos(rot), sr = std::sin(rot);
	const int npos = snx * sny;
	std::vector<float> pos(2 * (size_t)npos);
	for (int iy = 0; iy < sny; iy++)
		for (int ix = 0; ix < snx; ix++) {
			const size_t p = (size_t)iy * snx + ix;
			pos[2 * p] = offx + cr * stx * (float)ix - sr * sty * (float)iy;
			pos[2 * p + 1] = offy + cr * sty * (float)iy + sr * stx * (float)ix;
		}

	// run
	const int nd = GetDetetionSliceNum(), ndet = (int)ann.size();
	std::vector<float> out((size_t)npos * nd * ndet);
	JMS_SetScanBatch(64);
	const auto t0 = std::chrono::steady_clock::now();
	const int e = JMS_ScanGPU(npos, pos.data(), 0.f, nrep, nullptr, out.data(), nullptr, 0);
	const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
	if (e) {
		std::fprintf(stderr, "Error (jmsbench): JMS_ScanGPU returned %d\n", e);
		return 1;
	}
	// one file per detector: float [plane][scan y][scan x]
	std::vector<float> img((size_t)nd * npos);
	for (int j = 0; j < ndet; j++) {
		for (int pl = 0; pl < nd; pl++)
			for (int p = 0; p < npos; p++) img[(size_t)pl * npos + p] = out[((size_t)p * nd + pl) * ndet + j];
		const std::string f = out_file + "_" + ann[j].name + ".bin";
		std::ofstream os(f, std::ios::binary | std::ios::trunc);
		if (!os) return fail("cannot write ", f);
		os.write(reinterpret_cast<const char*>(img.data()), sizeof(float) * img.size());
	}
	std::printf("jmsbench: %d x %d scan, %d repeats, %d slices on %d x %d, %d planes x %d detectors: %.3f s "
		"(%.0f multislice steps/s)\n", snx, sny, nrep, nobj, nx, ny, nd, ndet, sec,
		(double)npos * nrep * nobj / sec);
	Cleanup();
	return 0;
}
