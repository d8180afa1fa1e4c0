/*
 * JProbeGen.h -- probe parameters of the CJMultiSlice class interface.
 *
 * CJProbeParams is the data class that CJMultiSlice::CalculateProbeWaveFourier
 * reads (the reference's src/JProbeGen.h:60-140).  Its data members, public
 * and protected, are declared in the reference's order and with its types, so
 * an object made by code compiled against the reference's header is read
 * correctly by this library.  Defaults (src/JProbeGen.cpp:53-80): 300 kV
 * wavelength 0.001969 nm, 25 mrad aperture with relative edge 0.03, no
 * aberrations; 24 aberrations (order <= 8), each an (x, y) pair in nm in the
 * order of the reference's aberration table (index 0 image shift, 1 defocus,
 * 2 twofold astigmatism, 3 coma, 4 threefold astigmatism, 5 spherical
 * aberration Cs, ...).  The probe-imaging part of the reference's CJProbeGen
 * class is not part of this library.  Implemented in libjms_b200.so.
 */
#ifndef JMS_B200_JPROBEGEN_H
#define JMS_B200_JPROBEGEN_H

#define _JPG_MESSAGE_LEN           2048 /* message length of the reference class */
#define _JPG_ABERRATION_ORDER_MAX  8    /* highest aberration order */

class CJProbeParams {
public:
	CJProbeParams(void);
	CJProbeParams(const CJProbeParams& src);
	~CJProbeParams(void);

	float m_wl;                    /* electron wavelength [nm] */
	float m_alpha;                 /* convergence semi-angle [mrad] */
	float m_alpha_rs;              /* relative aperture edge smoothness */
	float m_alpha_x0;              /* aperture centre [mrad] */
	float m_alpha_y0;
	float m_alpha_asym;            /* relative aperture asymmetry */
	float m_alpha_adir;            /* asymmetry direction [deg] */
	float m_btx;                   /* beam tilt [mrad] */
	float m_bty;
	float m_source_width;          /* source size (HWHM) [nm], not used by the wave calculation */
	int m_source_shape;            /* 0 point, 1 Gaussian, 2 Cauchy, 3 disk; not used by the wave */
	float m_fspread_width;         /* focus spread [nm], not used by the wave calculation */
	float m_fspread_kernel_width;  /* relative focus-spread kernel width */
	int m_fspread_kernel_samples;  /* focus-spread kernel samples */
	float* m_abrr_coeff;           /* 2 x GetAberrationNum() coefficients (x, y) [nm] */

protected:
	char m_msg[_JPG_MESSAGE_LEN];
	int m_abrr_num;

public:
	/* copies the data (aberrations up to the shorter table) */
	void operator=(const CJProbeParams& other);
	/* equal data and aberration tables */
	bool operator==(const CJProbeParams& other) const;
	/* number of aberrations in the table (24) */
	int GetAberrationNum(void);
	/* sets m_wl from the electron energy [keV]; returns it */
	float SetProbeEkV(float ekv);
};

#endif /* JMS_B200_JPROBEGEN_H */
