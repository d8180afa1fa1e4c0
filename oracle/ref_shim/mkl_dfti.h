/*
 * mkl_dfti.h -- build shim (test infrastructure only).
 *
 * Declares the subset of Intel MKL's public DFTI C API that the reference's
 * CJFFTMKLcore calls (src/JFFTMKLcore.cpp:68,129-142,176,196,213,233), bound
 * to the MKL 2024.2 copy inside PyTorch's libtorch_cpu.so.
 *
 * The reference passes the dimension list as an int array
 * (src/JFFTMKLcore.cpp:111-129), which matches MKL_LONG only on Windows'
 * LLP64 model.  On LP64 Linux the md descriptor wants 64-bit lengths, so the
 * DftiCreateDescriptor overloads below widen the int list before calling MKL.
 * Only single precision is used by the reference (DFTI_SINGLE).
 */
#pragma once

#ifndef MKL_LONG
#define MKL_LONG long
#endif

typedef struct DFTI_DESCRIPTOR* DFTI_DESCRIPTOR_HANDLE;

/* configuration values (public MKL enumeration) */
enum DFTI_CONFIG_VALUE {
	DFTI_COMMITTED = 30,
	DFTI_UNCOMMITTED = 31,
	DFTI_COMPLEX = 32,
	DFTI_REAL = 33,
	DFTI_SINGLE = 35,
	DFTI_DOUBLE = 36
};

/* error classes (public MKL enumeration, first entry only) */
enum DFTI_ERROR_CLASS {
	DFTI_NO_ERROR = 0
};

extern "C" {
MKL_LONG DftiCreateDescriptor_s_1d(DFTI_DESCRIPTOR_HANDLE*, enum DFTI_CONFIG_VALUE, MKL_LONG);
MKL_LONG DftiCreateDescriptor_s_md(DFTI_DESCRIPTOR_HANDLE*, enum DFTI_CONFIG_VALUE, MKL_LONG, MKL_LONG*);
MKL_LONG DftiCommitDescriptor(DFTI_DESCRIPTOR_HANDLE);
MKL_LONG DftiComputeForward(DFTI_DESCRIPTOR_HANDLE, void*, ...);
MKL_LONG DftiComputeBackward(DFTI_DESCRIPTOR_HANDLE, void*, ...);
MKL_LONG DftiFreeDescriptor(DFTI_DESCRIPTOR_HANDLE*);
char* DftiErrorMessage(MKL_LONG);
MKL_LONG DftiErrorClass(MKL_LONG, MKL_LONG);
}

/* multi-dimensional descriptor from an int length list */
static inline MKL_LONG DftiCreateDescriptor(DFTI_DESCRIPTOR_HANDLE* h, enum DFTI_CONFIG_VALUE prec,
	enum DFTI_CONFIG_VALUE domain, MKL_LONG dim, int* sizes)
{
	MKL_LONG lsz[8];
	if (prec != DFTI_SINGLE || dim < 1 || dim > 8 || sizes == 0) return 1;
	for (MKL_LONG i = 0; i < dim; i++) lsz[i] = (MKL_LONG)sizes[i];
	return DftiCreateDescriptor_s_md(h, domain, dim, lsz);
}

/* one-dimensional descriptor from a scalar length */
static inline MKL_LONG DftiCreateDescriptor(DFTI_DESCRIPTOR_HANDLE* h, enum DFTI_CONFIG_VALUE prec,
	enum DFTI_CONFIG_VALUE domain, MKL_LONG dim, int length)
{
	if (prec != DFTI_SINGLE || dim != 1) return 1;
	return DftiCreateDescriptor_s_1d(h, domain, (MKL_LONG)length);
}
