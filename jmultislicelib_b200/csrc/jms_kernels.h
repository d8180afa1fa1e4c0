// jms_kernels.h -- device-side entry points of the fused multislice passes.
//
// The multislice step of the reference (src/JMultiSlice.cpp:4590-4651:
// [readout psi(k)] -> IFT -> [readout psi(r)] -> x t -> FT -> x P) is run as two
// fused global passes over a batch of waves held [wave][ny][nx] (x fastest):
//
//   column pass  (one CTA = a tile of columns):  IFT_y -> [image readout]
//                -> x t -> FT_y
//   row pass     (one CTA = a tile of rows):     FT_x  -> x P (band limit is
//                part of P) -> [Fourier readout] -> IFT_x
//
// Between the passes the wave is half transformed (x real / y Fourier after
// the row pass, y Fourier / x real after the column pass), so each step reads
// and writes the wave exactly twice.  An entry row pass applies the probe
// offset and the entrance-plane readout, then IFT_x; an exit column pass
// provides the exit-plane image readout.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace jms {

constexpr int kMaxDet = 8;          // integrating detectors fused into one pass

struct PassArgs {
	float2* work = nullptr;         // [nwave][ny][nx] working waves
	long long wstride = 0;          // elements between consecutive waves
	int nx = 0, ny = 0, nwave = 0;
	const float2* twx = nullptr;    // exp(-2 pi i k / nx), k < nx
	const float2* twy = nullptr;    // exp(-2 pi i k / ny), k < ny
	// multiplicative operand of this step
	const float2* mul = nullptr;    // column pass: grating [npgy][npgx]; row pass: propagator [ny][nx]
	int npgx = 0, npgy = 0;
	// readout at this plane (-1 = none)
	int plane = -1;
	int ndetslc = 0;
	float weight = 1.f;
	int ndet = 0;                   // integrating detectors (0 = off)
	const float* det = nullptr;     // [ndet][ny][nx], masks folded in
	float* partial = nullptr;       // [nwave][ndetslc][ndet][nblk] per-CTA sums
	int nblk = 0;                   // row-pass CTAs per wave
	long long chan_wstride = 0;     // per-wave stride of full-size channels (0 = one shared channel)
	float* dif = nullptr;           // Fourier channels [ndetslc][ny][nx]
	float* dif_avg = nullptr;
	float2* wff = nullptr;
	float2* wff_avg = nullptr;
	float* img = nullptr;           // real-space channels [ndetslc][ny][nx]
	float* img_avg = nullptr;
	float2* wfr = nullptr;
	float2* wfr_avg = nullptr;
	float* bin_out = nullptr;       // [nwave][nby][nbx] unscrambled, binned |psi(k)|^2
	int bin = 1, nbx = 0, nby = 0;
	int bin_plane = -1;             // plane at which the binned pattern is taken
	int descan_x = 0, descan_y = 0; // integer-pixel diffraction descan of the Fourier readout
	// column pass: cyclic shift (plas_x, plas_y) pixels of the spectrum after
	// the forward transform (plasmon scattering, CShift2d), applied as the
	// real-space ramp exp(2 pi i (plas_x x / nx + plas_y y / ny)) with x t
	int plas_x = 0, plas_y = 0;
	const int* plas_w = nullptr;    // [nwave][2] per-wave shifts of this slice (replaces plas_x / plas_y)
	// column pass: per-wave element offsets of each wave's grating from mul
	// (waves of different frozen-phonon configurations in one launch);
	// nullptr = the grating at mul for every wave
	const int* mul_w = nullptr;
	// > 0: wave b is probe position b % wave_pos (several configurations of
	// the positions in one launch): binned patterns go to the position
	int wave_pos = 0;
	int store = 1;                  // row pass: 0 = stop after the readout (last slice)
	// Band of live Fourier rows: row ky (scrambled index) can be nonzero only
	// if ky <= k1 or ky >= k2.  Propagators vanish outside their band limit,
	// so after x P the other rows are exactly zero: the row pass skips them
	// (row_k1/row_k2, band of its propagator), the column pass reads them as
	// zero (in_k1/in_k2) and does not store them (out_k1/out_k2, band of the
	// next row pass).  k1 = ny - 1 marks all rows live.  For the entry pass,
	// row_k1/row_k2 is the band of its source's live rows.
	int row_k1 = 1 << 30, row_k2 = 1 << 30;
	int in_k1 = 1 << 30, in_k2 = 1 << 30;
	int out_k1 = 1 << 30, out_k2 = 1 << 30;
	// entry pass source: wav0 (nullptr = the work buffer); with shift set, wav0
	// is the incident wave and each wave b gets its own probe offset
	const float2* wav0 = nullptr;   // [ny][nx] Fourier space
	const double* shift = nullptr;  // [nwave][4]: dx/a, dy/b, fz/a^2, fz/b^2 (phase in turns)
	const float* cppl = nullptr;    // constant phase plate [ny][nx] or nullptr
	int ibtx = 0, ibty = 0;         // beam tilt in Fourier pixels
};

// Line plans: every supported length n has one or more candidate plans
// (jms_sizes.h); the row/entry passes use the plan chosen for nx, the
// column/exit passes the plan chosen for ny.  Index 0 is a length's default.
struct PlanOps {
	int n;
	const char* name;
	int (*row_blocks)(int ny);                              // row-pass CTAs per wave
	cudaError_t (*entry)(const PassArgs&, cudaStream_t);    // entry row pass
	cudaError_t (*row)(const PassArgs&, cudaStream_t);      // row pass
	cudaError_t (*col)(const PassArgs&, cudaStream_t);      // column pass
	cudaError_t (*exit)(const PassArgs&, cudaStream_t);     // exit column pass
};
int plan_count(int n);
const PlanOps* plan_get(int n, int idx);
inline bool pass_supported(int n) { return plan_count(n) > 0; }

// Tensor-core forms of the row and column passes (jms_tc.cu) for line lengths
// 256, 512, 1024 and 2048: prec 1 = BF16 hi+lo operands, 2 = FP16 hi+lo, FP32
// accumulation.  No readout; the column pass needs a grating of the grid size
// and no plasmon shift.  *err is set to 1 if a tensor-core wait ran out.
bool tc_supported(int n);
// builds the DFT-matrix tables of the tensor-core passes on the current device
// (once per device, before the first pass; synchronises s)
cudaError_t tc_prepare(cudaStream_t s);
cudaError_t launch_tc_row(const PassArgs& p, int prec, int* err, cudaStream_t s);
cudaError_t launch_tc_col(const PassArgs& p, int prec, int* err, cudaStream_t s);

// det_int[w][plane][d] += weight * sum_blk partial[w][plane][d][blk] (FP64);
// with wave_pos > 0 the waves w = p + k wave_pos (k = 0, 1, ...) are summed
// into position p, in that order (deterministic)
cudaError_t launch_finalize(const float* partial, int nwave, int ndetslc, int ndet, int nblk, float weight,
	double* det_int, cudaStream_t s, int wave_pos = 0);

// sh_w[w] = sh[w % npos] (4 doubles each), w < nwave: per-wave probe offsets
// of several configurations of the same positions
cudaError_t launch_gather_shift(double* sh_w, const double* sh, int npos, int nwave, cudaStream_t s);

// shift[i] = (dx/a, dy/b, fz/a^2, fz/b^2) from pos[i] = (dx, dy) [nm]
cudaError_t launch_make_shift(double* d_shift, const float* d_pos, int npos, double a, double b, double fz,
	cudaStream_t s);

// Integrated-detector readout of nwave Fourier-space waves [nwave][ny][nx]
// that allocates nothing: its partial sums live in a fixed file-scope device
// array (jms_noalloc.cu).  out[w][d] = sum_k |wav_w(k)|^2 det_d(k) (FP64,
// overwritten).  Returns 0, 131 (needs more than noalloc_capacity() partial
// sums), 132 (no device address for the array) or 133 (launch error).
int launch_readout_noalloc(const float2* wav, int nwave, int nx, int ny, const float* det, int ndet, double* out,
	cudaStream_t s);
int noalloc_capacity();

// out[i] += c (gm[i] - g1[i]), i < n: the control-variate correction of the
// multi-fidelity scan (JMS_ScanMultiFidelityDevice)
cudaError_t launch_cv_combine(double* out, const double* g1, const double* gm, long long n, double c, cudaStream_t s);

// out[i] = |in[i]|^2, i < n
cudaError_t launch_abs2(float* out, const float2* in, long long n, cudaStream_t s);

// drop-in OffsetIncomingWave: out = wav0(k - tilt) * exp(-i(2 pi turns + cppl))
cudaError_t launch_offset(float2* out, const float2* wav0, int nx, int ny, const double* shift_host4,
	const float* cppl, int ibtx, int ibty, cudaStream_t s);

} // namespace jms
