/*
 * jms_b200.h -- C ABI of the B200 multislice library (libjms_b200.so).
 *
 * Drop-in for the GPU multislice path of JMultiSliceLib's flat interface
 * (src/JMultiSliceLib.h:108-380): the same symbol names, argument meanings,
 * flag values, result layouts and integer error codes (0 = success), exported
 * as plain extern "C" without __stdcall/__declspec.  Each declaration names
 * the reference entry point it replaces (src/JMultiSliceLib.h:<line>).
 *
 * Conventions
 *   - complex arrays are interleaved float pairs (re, im), row-major [ny][nx]
 *     with x fastest, Fourier space in scrambled (FFT) order, as fcmplx in the
 *     reference;
 *   - C++ references of the reference interface become pointers here
 *     (GetGridSize, GetGPUStats, CalculateRingDetector's msklen), the
 *     std::string profile name becomes const char*, and CJProbeParams*
 *     becomes JMSProbeParams* (its public data members, same order);
 *   - whichcode: 1 = CPU, 2 = GPU.  This library has no CPU code path: any call
 *     with the CPU bit set returns 1 and does nothing (CPUMultislice,
 *     SetIncomingWaveCPU and ClearDetMem_h always return 1);
 *   - all device memory is owned by the library; inputs are copied at Set*,
 *     results are copied out by GetResult / GetAvgResult;
 *   - one library instance (like the reference's static CJMultiSlice) serves
 *     the flat calls; calls are not re-entrant.
 */
#ifndef JMS_B200_H
#define JMS_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* flag values (src/JMultiSlice.h:126-149) */
#define JMS_CODE_CPU            1
#define JMS_CODE_GPU            2
#define JMS_DETECT_INTEGRATED   1
#define JMS_DETECT_IMAGE        2
#define JMS_DETECT_DIFFRACTION  4
#define JMS_DETECT_WAVEREAL     8
#define JMS_DETECT_WAVEFOURIER  16
#define JMS_DETECT_IMAGE_AVG    32
#define JMS_DETECT_DIFFR_AVG    64
#define JMS_DETECT_WAVER_AVG    128
#define JMS_DETECT_WAVEF_AVG    256
#define JMS_ACCMODE_NONE        0
#define JMS_ACCMODE_INTEGRATE   1

/* public data of CJProbeParams (src/JProbeGen.h:60-94), same order */
typedef struct JMSProbeParams {
	float m_wl;                 /* wavelength [nm] (replaced by the library's) */
	float m_alpha;              /* convergence semi-angle [mrad] */
	float m_alpha_rs;           /* relative aperture edge smoothness */
	float m_alpha_x0, m_alpha_y0; /* aperture centre [mrad] */
	float m_alpha_asym;         /* relative aperture asymmetry */
	float m_alpha_adir;         /* asymmetry direction [deg] */
	float m_btx, m_bty;         /* beam tilt [mrad] */
	float m_source_width;       /* unused by the wave calculation */
	int m_source_shape;         /* unused by the wave calculation */
	float m_fspread_width;      /* unused by the wave calculation */
	float m_fspread_kernel_width; /* unused by the wave calculation */
	int m_fspread_kernel_samples; /* unused by the wave calculation */
	float* m_abrr_coeff;        /* 2 * 24 aberration coefficients (x, y) [nm] */
} JMSProbeParams;

/* ---- basic interface ---------------------------------------------------- */
float GetJMSVersion(void);                       /* src/JMultiSliceLib.h:111 */
int SetJMSDebugLevel(int debuglevel);            /* src/JMultiSliceLib.h:114 */
void SeedRngEx(int rngseed);                     /* src/JMultiSliceLib.h:123 */

/* ---- physics interface ---------------------------------------------------- */
float SetHighTension(float ht);                  /* src/JMultiSliceLib.h:129 */
float GetHighTension(void);                      /* src/JMultiSliceLib.h:132 */
float GetWaveLength(void);                       /* src/JMultiSliceLib.h:135 */
void SetSupercellSize(float* a0);                /* src/JMultiSliceLib.h:138 */
void SetSupercellSizeABC(float a, float b, float c); /* src/JMultiSliceLib.h:141 */
void SetSliceThickness(int islc, float fthickness);  /* src/JMultiSliceLib.h:146 */
void DiffractionDescan(int bActivate);           /* src/JMultiSliceLib.h:149 (bool) */
void SetPlasmonMC(int bActivate, float fq_e, float fq_c, float fmfp, unsigned int nexmax); /* :152; bulk plasmon
	Monte-Carlo: q_e, q_c [1/nm], mean free path [nm], max. excitations; the pixel shift of each slice is drawn
	on the host from the library RNG after the variant draw (CJPlasmonMC::ScatGridMC) and applied in the
	column pass */
void SetDiffractionDescanN(int whichcode, int ndescanx, int ndescany, int iThread);       /* :160 */
void SetDiffractionDescan(int whichcode, float descanx, float descany, int iThread);     /* :168 */
void SetDiffractionDescanMRad(int whichcode, float descanx, float descany, int iThread); /* :176 */

/* ---- numerics interface --------------------------------------------------- */
void SetGridSize(int nx, int ny);                /* src/JMultiSliceLib.h:183 */
void GetGridSize(int* nx, int* ny);              /* src/JMultiSliceLib.h:186 (int& -> int*) */
int GetDetetionSliceNum(void);                   /* src/JMultiSliceLib.h:189 */
int GetDetNum(void);                             /* src/JMultiSliceLib.h:192 */
int GetCPUNum(void);                             /* src/JMultiSliceLib.h:195 */
int GetGPUNum(void);                             /* src/JMultiSliceLib.h:198 */
int GetGPUName(int idev, char* name);            /* src/JMultiSliceLib.h:201 (name: 256 bytes) */
int GetCurrentGPU(void);                         /* src/JMultiSliceLib.h:204 */
int SetCurrentGPU(int idev);                     /* src/JMultiSliceLib.h:207 */
int GetGPUStats(int idev, int* iCMajor, int* iCMinor, int* iMaxThread, int64_t* CUDAmemtotal,
	int64_t* CUDAmemfree);                       /* src/JMultiSliceLib.h:210 (refs -> pointers) */
int GetUnscrambleHash(unsigned int* phash);      /* src/JMultiSliceLib.h:220 */
float GetImageAveragingWeight(int whichcode, int iThread); /* src/JMultiSliceLib.h:223 */
float GetWaveAveragingWeight(int whichcode, int iThread);  /* src/JMultiSliceLib.h:226 */

/* ---- setup interface ------------------------------------------------------ */
int PhaseGratingSetup(int whichcode, int nx, int ny, int nslc, int nvarmax, int* nslcvar); /* :231 */
int ObjectSliceSetup(int nobjslc, int* objslc);  /* src/JMultiSliceLib.h:234 */
int PropagatorSetup(int whichcode, int npro, int* proidx); /* src/JMultiSliceLib.h:237 */
int DetectorSetup(int whichcode, int ndetper, int ndetint, int imagedet, int nthreads_CPU); /* :240; ndetint <= 8 */
int InitCore(int whichcode, int nCPUthreads);    /* src/JMultiSliceLib.h:243 */
int SetIncidentWave(int whichcode, float* wav);  /* src/JMultiSliceLib.h:246 */
int SetIncidentWavePhaseplate(int whichcode, float* ppl, int bTranspose); /* src/JMultiSliceLib.h:249 */
int ZeroIncidentWavePhaseplate(int whichcode);   /* src/JMultiSliceLib.h:252 */
int SetSlicePhaseGratings(int whichcode, int islc, int nvar, float* pgr); /* src/JMultiSliceLib.h:255 */
int SetPropagatorData(int whichcode, int ipro, float* pro); /* src/JMultiSliceLib.h:258 */
int SetDetectorData(int whichcode, int idet, float* det, int msklen, int* msk); /* src/JMultiSliceLib.h:261 */
int SetGPUPgrLoading(int npgrload);              /* src/JMultiSliceLib.h:266 (accepted, gratings stay on the device) */
int ResetImageAveraging(int whichcode, int iThread); /* src/JMultiSliceLib.h:269 */
int ResetWaveAveraging(int whichcode, int iThread);  /* src/JMultiSliceLib.h:272 */

/* ---- calculation interface ------------------------------------------------ */
int CalculateProbeWaveFourier(JMSProbeParams* prm, float* wav); /* src/JMultiSliceLib.h:280 */
int SetIncomingWaveGPU(float* wav, int bTranspose);   /* src/JMultiSliceLib.h:286 */
int SetIncomingWaveCPU(float* wav, int bTranspose, int iThread); /* src/JMultiSliceLib.h:293; returns 1 */
int CalculatePropagator(float fthick, float otx, float oty, float* pro, int ntype); /* src/JMultiSliceLib.h:303 */
int CalculateRingDetector(float beta0, float beta1, float phi0, float phi1, float theta0x, float theta0y,
	const char* sdsprofile, float* det, int* msklen, int* msk, int kmom1); /* src/JMultiSliceLib.h:318 */
int OffsetIncomingWave(int whichcode, float dx, float dy, float dz, int iThread, int ibtx, int ibty); /* :326 */
int CPUMultislice(int islc0, int accmode, float weight, int iThread); /* src/JMultiSliceLib.h:333; returns 1 */
int GPUMultislice(int islc0, int accmode, float weight); /* src/JMultiSliceLib.h:339 */
int GetResult(int whichcode, int whichresult, float* dst, int iThread); /* src/JMultiSliceLib.h:346 */
int GetAvgResult(int whichcode, int whichresult, float* dst, float* wgt, int iThread); /* src/JMultiSliceLib.h:354 */
int ClearDetMem_h(int iThread);                  /* src/JMultiSliceLib.h:357; returns 1 */
int ClearDetMem_d(void);                         /* src/JMultiSliceLib.h:363 */

/* ---- cleanup interface ---------------------------------------------------- */
int Cleanup(void);                               /* src/JMultiSliceLib.h:375 */
void FreeLibMem(void);                           /* src/JMultiSliceLib.h:380 */

/* ---- additions (no counterpart in the reference interface) ---------------- */
/* Runs the library's kernels on the given CUDA stream (cudaStream_t passed as
 * void*; NULL selects the library's own stream). */
int JMS_SetStream(void* stream);
/* Batched STEM scan on the current setup: npos probe positions pos[2*i] = dx,
 * pos[2*i+1] = dy [nm] (defocus dz [nm] for all), each averaged over npass
 * frozen-phonon passes (weight 1/npass).  varseq: npass x nobjslc variant
 * indices, or NULL to draw them like GPUMultislice.  Host buffers:
 * out_int [npos][ndetslc][ndet]; out_bin [npos][ny/bin][nx/bin] unscrambled
 * exit-plane diffraction binned bin x bin (NULL to skip). */
int JMS_ScanGPU(int npos, const float* pos, float dz, int npass, const int* varseq, float* out_int,
	float* out_bin, int bin);
/* The same with device buffers, asynchronous on the library stream;
 * d_out_int is double [npos][ndetslc][ndet] and is accumulated into. */
int JMS_ScanGPUDevice(int npos, const float* d_pos, float dz, int npass, const int* varseq, double* d_out_int,
	float* d_out_bin, int bin);
/* Probe positions processed together in one pass sequence (default 32). */
int JMS_SetScanBatch(int nwave);
/* Frozen-phonon configurations in one launch (no counterpart in the
 * reference, whose GPUMultislice runs one wave per call,
 * src/JMultiSlice.cpp:4513-4677).  When a scan has more than one pass, fewer
 * positions than the scan batch and no plasmon paths, several configurations
 * of its positions share each launch sequence (without a variant sequence the
 * library draws all configurations first, in the sequential order): each
 * wave reads its own configuration's grating, and the detector sums and
 * binned patterns of a position collect its waves in a fixed order.  on = 1
 * (default) allows it, 0 runs one launch sequence per configuration.  Scans
 * enqueued during a stream capture always take the sequential form. */
int JMS_SetPassFusion(int on);
/* Multi-fidelity frozen-phonon scan (no counterpart in the reference, which
 * averages every configuration at full cost, src/JMultiSlice.cpp:4513-4677
 * per pass).  Estimates the npass-configuration average of context ctx_full
 * from ONE full pass (configuration 0 of varseq) and npass passes of context
 * ctx_low, a coarser grid of the same specimen, probe, detectors and slices:
 *   est = f(c0) - (g(c0) - mean_c g)       (control variate, coefficient 1)
 * The estimate is unbiased.  Its error is that of f - g across the
 * configurations; for detectors inside the coarse grid's band limit the
 * phonon fluctuations of f and g agree closely (ratio 1.0000 +- 1e-4 and
 * correlation^2 = 1 - 1e-7 measured for 512^2 against 256^2).  Detectors
 * outside it get g = 0, so the estimate is the single full pass there.
 * varseq: npass x nobjslc variant indices (required; both contexts use the same
 * configurations).  Device form: d_pos [npos][2] nm and d_out_int double
 * [npos][ndetslc][ndet] on the device (d_out_int overwritten).  The two
 * contexts run concurrently on their own streams, and the call returns
 * without waiting.  d_pos must be ready for both streams.  Successive device
 * calls may be issued back to back: their coarse sums alternate between two
 * halves of the coarse context's scratch, each cleared only after the combine
 * that last read it (an event on the full context's stream).  Host form: host
 * buffers, returns after the copy back.  Returns 0, 1 (bad arguments or
 * context), 2 (a context lacks its stream / setup), 3 (the contexts' slice or
 * detector counts differ), 4 (scratch allocation), 5 (CUDA error), or an error
 * of the scans. */
int JMS_ScanMultiFidelityDevice(int ctx_full, int ctx_low, int npos, const float* d_pos, float dz, int npass,
	const int* varseq, double* d_out_int);
int JMS_ScanMultiFidelity(int ctx_full, int ctx_low, int npos, const float* pos, float dz, int npass,
	const int* varseq, float* out_int);
/* Kernel launches issued by the library so far. */
long long JMS_KernelLaunches(void);
/* Per-pass device timing: while on, each column and row pass launch is
 * bracketed by CUDA events on the library stream; JMS_PassTiming returns the
 * summed milliseconds and launch counts since the last JMS_SetPassTiming. */
void JMS_SetPassTiming(int on);
int JMS_PassTiming(double* ms_col, long long* n_col, double* ms_row, long long* n_row);
/* Integrated detectors of caller-provided waves, allocating no memory.  No
 * counterpart in the reference interface.  For callers that must not have
 * the library allocate device memory while they run (a fixed memory pool
 * owns the GPU, a real-time loop cannot afford the device synchronisation of
 * cudaMalloc/cudaFree, or the footprint must stay fixed after start-up).
 * d_wav: device, nwave Fourier-space waves [nwave][ny][nx] (interleaved
 * float pairs, the grid of the current setup); d_out: device, double
 * [nwave][ndet], overwritten with sum_k |psi(k)|^2 D_d(k) for the detectors
 * of the current setup (masks applied).  stream: cudaStream_t or NULL for the
 * library stream.  The per-CTA partial sums live in one fixed file-scope
 * device array of 65536 floats (256 KiB per GPU, held until the process
 * ends); calls needing more than nwave * ndet * ceil(ny / 8) <= 65536 are
 * refused with 131.  All calls share that array, so calls that overlap on
 * the GPU race; JMS_ReadoutDetAvg with JMS_DETECT_INTEGRATED uses the same
 * array on the library stream, so serialise it with calls of this function
 * on other streams.  The first call on a device looks up the array's address
 * (cudaGetSymbolAddress) with that device current: make it before any stream
 * capture.  The address is kept per device and CUDA context; a call under a
 * different context of the device looks it up again.  Returns 0, 1 (bad
 * arguments), 2 (setup incomplete), 131, 132 (address lookup failed) or 133
 * (launch failed). */
int JMS_ReadoutDetectorsNoAlloc(const float* d_wav, int nwave, double* d_out, void* stream);
/* Line-plan autotuner (no counterpart in the reference): times each candidate
 * FFT plan of nx (row passes) and ny (column passes) on nwave waves of the
 * current setup (reps launches each, CUDA events) and keeps the fastest for
 * this and later setups of the same lengths in the process.  Outputs (may be
 * NULL): average ms per launch of the chosen plans and their indices. */
int JMS_Autotune(int nwave, int reps, float* ms_row, float* ms_col, int* irow, int* icol);
/* Chooses the row / column plans by index (0 = default); 1 if out of range. */
int JMS_SelectPlans(int irow, int icol);
/* Number of candidate plans for line length n (0 = length not supported). */
int JMS_PlanCount(int n);
/* Name of the plan in use for axis 0 (rows, nx) or 1 (columns, ny). */
int JMS_PlanName(int axis, char* name, int len);
/* 1 if both grid lengths are supported by the fused passes. */
int JMS_GridSupported(int nx, int ny);
/* Arithmetic of the line transforms (no counterpart in the reference, whose
 * GPU path is cuFFT in FP32, src/JFFTCUDAcore.cpp:299-336): 0 = FP32 passes
 * (default); 1 = tensor-core passes, each radix-16/32/64 stage a
 * DFT-matrix product with BF16 hi+lo operands and FP32 accumulation; 2 = the
 * same with FP16 hi+lo operands (power-of-two scaled per tile).  The
 * tensor-core passes serve the slices without readout on grids whose lengths
 * are 256, 512, 1024 or 2048; readout slices, sub-frame gratings, plasmon
 * shifts and other lengths run the FP32 passes.  Returns 0, or 1 for a mode
 * out of range. */
int JMS_SetPrecision(int mode);
int JMS_GetPrecision(void);
/* 1 if a tensor-core pass found its matrix products unfinished after its
 * bounded wait (about a second) since the last call, else 0 (-1 on a CUDA
 * error); synchronises the library stream and clears the flag. */
int JMS_TcStatus(void);
/* Tensor-core pass launches issued by the library so far. */
long long JMS_TcLaunches(void);

/* Detector readouts of the averaged wave functions: the public method
 * CJMultiSlice::ReadoutDetAvg (src/JMultiSlice.h:935, .cpp:2667-2945), GPU
 * branch, which the reference's flat interface does not export.  whichresult
 * JMS_DETECT_INTEGRATED: dst[idetslc * ndet + idet] = sum_k |<psi(k)>|^2 D(k)
 * over the averaged Fourier-space waves (WAVEF_AVG); JMS_DETECT_IMAGE /
 * JMS_DETECT_DIFFRACTION: dst [ndetslc][ny][nx] = |<psi(r)>|^2 / |<psi(k)>|^2
 * of the averaged real-space / Fourier-space waves.  Each needs its detection
 * flag and the averaged wave; *weight = the wave averaging weight (the sums
 * are not divided by it).  Returns 0 (also when there is nothing to read),
 * 1 for the CPU code, or 21-23 / 121-122 on device errors. */
int JMS_ReadoutDetAvg(int whichcode, int whichresult, float* dst, float* weight);

/* ---- contexts and CUDA graphs -------------------------------------------
 * A context is one library instance (grid, setup, device buffers, stream) --
 * what a separate CJMultiSlice object is in the reference's C++ interface.
 * Context 0 is the default one behind the flat functions; JMS_CreateContext
 * returns the id of a new one, JMS_SelectContext(id) directs the flat calls
 * of the calling host thread to it (returns the previous id, -1 for an
 * unknown id), JMS_DestroyContext(id) frees it (id > 0).  Contexts of
 * different grid sizes run their scans concurrently: each works on its own
 * stream (created by InitCore), and JMS_ScanGPUDevice only enqueues. */
int JMS_CreateContext(void);
int JMS_SelectContext(int id);
int JMS_DestroyContext(int id);
/* Stream capture of the work that the listed contexts enqueue between
 * JMS_GraphBegin and JMS_GraphEnd into one CUDA graph (fork / join over the
 * contexts' streams).  JMS_GraphEnd returns a handle >= 1 (negative on
 * failure).  A graph replays exactly the captured work: kernel arguments,
 * variant sequences and the device buffers they read, whose contents the
 * caller may refresh between launches (positions); synchronous calls,
 * buffer growth, pass timing and plasmon draws are not allowed while
 * capturing, so run each workload once before capturing it.
 * JMS_GraphLaunch(handle, stream or NULL, wait). */
int JMS_GraphBegin(int nctx, const int* ctx);
int JMS_GraphEnd(void);
int JMS_GraphLaunch(int handle, void* stream, int wait);
int JMS_GraphDestroy(int handle);

/* ---- EMS slice files (.sli) ----------------------------------------------
 * Phase-grating files of Dr. Probe / EMS as the reference's bench driver reads
 * them (test/JMSBench1/prm_slice_file_info.h:60-150, prm_slice_file_info.cpp
 * load_ems_header, prm_slice.cpp load_ems_data): 8192-byte header, nvar
 * complex64 gratings [nvar][ny][nx] at data_offset.  Files of the other byte
 * order are detected (first word outside [0, 16384]) and swapped on input. */
typedef struct JMSSliHeader {
	int nx, ny;                 /* grid */
	int nvar;                   /* number of variants (1 for old header versions) */
	int content;                /* 0 phase grating, 1 potential */
	unsigned int version;       /* extended header version */
	unsigned int data_offset;   /* byte offset of the gratings */
	unsigned int table_offset;  /* byte offset of the atom table */
	float thickness;            /* slice thickness [nm] */
	float ekv;                  /* beam energy [keV] */
	float sx, sy;               /* slice size [nm] */
	int swapped;                /* 1 if the file has the other byte order */
	char title[41];             /* slice title (40 chars + NUL) */
} JMSSliHeader;
/* Returns 0, 1 (bad arguments), 2 (cannot open), 3 (short header), 4 (invalid header). */
int JMS_SliReadHeader(const char* path, JMSSliHeader* hdr);
/* Reads the nvar gratings into pgr (2 * nx * ny * nvar floats); 5 = short data. */
int JMS_SliReadData(const char* path, float* pgr);
/* Writes a slice file (header version 2020052801, data at 8192, empty atom
 * table) from hdr (nx, ny, nvar, content, thickness, ekv, sx, sy, title) and
 * pgr; 6 = write error. */
int JMS_SliWrite(const char* path, const JMSSliHeader* hdr, const float* pgr);
/* Loads a slice file's gratings as the variants of structure slice islc of
 * the GPU setup (SetSlicePhaseGratings); 7 = grid of the file differs from
 * the grating grid of PhaseGratingSetup. */
int JMS_SliLoadSlice(const char* path, int islc);

/* ---- control-variate surrogate network (no counterpart in the reference) ---
 * Building blocks of the small convolutional surrogate used as a control
 * variate for frozen-phonon averaging (jmultislicelib_b200/surrogate.py):
 * BF16 activations and weights, FP32 accumulation, FP32 gradients.  All
 * pointers are device pointers, stream may be NULL.  Layouts: activations
 * [B][C][H][W], conv weights [Co][Ci][3][3] (3x3, stride 2, padding 1),
 * linear weights [O][C].  Return 0, or 2 for bad arguments, 1 for a launch
 * error. */
int JMS_NnConvForward(const void* x, const void* w, const float* bias, void* y, int B, int Ci, int H, int W, int Co,
	int relu, void* stream);
/* Backward of JMS_NnConvForward from dL/dy (before the ReLU mask, which is
 * taken from the stored output y): dx (may be NULL), dw, db. */
int JMS_NnConvBackward(const void* x, const void* w, const void* y, const float* dy, float* dx, float* dw, float* db,
	int B, int Ci, int H, int W, int Co, int relu, void* stream);
/* out[b][o] = bl[o] + sum_c wl[o][c] * mean over HW of h[b][c] (h BF16). */
int JMS_NnPoolLinearForward(const void* h, const float* wl, const float* bl, float* out, int B, int C, int HW, int O,
	void* stream);
int JMS_NnPoolLinearBackward(const void* h, const float* wl, const float* dout, float* dh, float* dwl, float* dbl,
	int B, int C, int HW, int O, void* stream);
/* Mean squared error over n values: dout = 2 (out - target) / n, *loss (may
 * be NULL) = mean (out - target)^2. */
int JMS_NnMseLoss(const float* out, const float* target, float* dout, float* loss, int n, void* stream);
/* One Adam step (step >= 1) on FP32 parameters p with moments m, v; writes a
 * BF16 copy to p_bf16 when given. */
int JMS_NnAdam(float* p, const float* g, float* m, float* v, void* p_bf16, int n, float lr, float b1, float b2,
	float eps, int step, void* stream);
int JMS_NnCastBf16(const float* src, void* dst, long long n, void* stream);
/* Surrogate inputs on the device: out [nconf][npos][nbins][win/pool][win/pool]
 * = the mean, over the object slices of each depth bin (nbins bins of
 * nobj / nbins consecutive slices, the first nobj % nbins one slice longer)
 * and over pool x pool pixel blocks, of the projected potential in the
 * win x win-pixel window centred on the probe pixel (periodic).  pot [ntype]
 * [nvar][ny][nx] float (potential of structure slice t, variant v); objslc
 * [nobj] structure slice of each object slice; var [nconf][nobj] variant of
 * each object slice per configuration; pix [npos][2] probe pixel (x, y).
 * Device pointers; returns 0, 2 for bad arguments, 1 for a launch error. */
int JMS_NnPatches(const float* pot, int ntype, int nvar, int nx, int ny, const int* objslc, int nobj, const int* var,
	int nconf, const int* pix, int npos, int nbins, int win, int pool, float* out, void* stream);

/* ---- on-device phase gratings (CJEElaSca, src/JEElaSca.h:98-273) --------
 * The 2-D projection mode of CJEElaSca::CalculatePhasegratingGPU
 * (src/JEElaSca.cpp:978-1159) run on the device: Fourier synthesis of the
 * projected potential from radial form-factor tables, inverse FFT,
 * t = exp(i sigma V) (phase reduced in FP64) and the 2/3 band limit.
 * JMS_PgrSetup: grid nx x ny over the orthorhombic cell a x b [nm]
 * (SetGrid / CStructure cell), beam energy [keV], thermal model (0 none,
 * 1 Debye-Waller factors inside the form factors, 2 QEP site displacements),
 * band limits of the potential (m_bwl_pot, reference default 0) and of the
 * grating (m_bwl_pgr, default 1).  Returns 0, 1 (bad arguments) or 8
 * (grid length without a line plan). */
int JMS_PgrSetup(int nx, int ny, float a, float b, float ekv, int thermal, int bwl_pot, int bwl_pgr);
/* Radial form factors of the atom types: ff [ntype][nk] complex (nm),
 * sample k at q = k * sk [1/nm] (the table CAtomType::CopyFormFactors returns,
 * src/Atoms.h:122-125), and Biso [nm^2] per type (QEP amplitudes; may be NULL). */
int JMS_PgrSetFormFactors(int ntype, int nk, float sk, const float* ff, const float* biso);
/* Stream of the generator's kernels; NULL (the default) runs them on the
 * current context's stream.  With a stream of its own, the generation of one
 * set of gratings can overlap the scans of the context's stream.  The caller
 * orders the two with events: a scan waits for the generation of the gratings
 * it reads, and a generation into grating variants waits for the scans still
 * reading them.  No reference counterpart (CJEElaSca's GPU path runs on the
 * default stream); returns 0. */
int JMS_PgrSetStream(void* stream);
/* ngr phase gratings of one structure slice: atoms [natom][5] = fractional
 * x, y, z in the cell, occupancy, type index; cz = slice thickness [nm].
 * Atoms closer than 0.05 nm share a site (CStructure::SetAtomSites,
 * src/Structure.cpp:441-491); under the QEP model every grating is a new draw
 * of the site displacements (SplitMix64 stream of seed, Box-Muller).  With
 * islc >= 0 the gratings become variants ivar0 .. ivar0 + ngr - 1 of
 * structure slice islc in the multislice setup (PhaseGratingSetup grid must
 * equal the generator grid); pgr (may be NULL) receives them as complex
 * [ngr][ny][nx].  Returns 0, 1 (setup incomplete), 2 (bad atom type or
 * occupancy), 3 (bad arguments), 4 (allocation), 5 (copy), 6/7 (kernels),
 * 9 (islc / ivar0 / grid do not match the grating setup). */
int JMS_PgrCalculate(int natom, const float* atoms, float cz, int ngr, unsigned long long seed, int islc, int ivar0,
	float* pgr);

#ifdef __cplusplus
}
#endif

#endif /* JMS_B200_H */
