/*
 * mkl.h -- build shim for compiling the reference JMultiSliceLib CPU path on
 * Linux (test infrastructure only; nothing in the product includes this).
 *
 * The reference's CJFFTMKLcore (src/JFFTMKLcore.h:48-49) includes <mkl.h> and
 * <mkl_dfti.h>.  No standalone MKL is installed here, but PyTorch's
 * libtorch_cpu.so carries Intel MKL 2024.2 and exports the DFTI entry points
 * (DftiCreateDescriptor_s_md, DftiComputeForward, ...).  This header declares
 * that public API subset so the reference's own JFFTMKLcore.cpp runs on the
 * real MKL DFT, linked from libtorch_cpu.so.
 *
 * It also provides the Windows CRT function memcpy_s used by
 * CJFFTMKLcore::CShift2d (src/JFFTMKLcore.cpp:309-319).
 */
#pragma once
#include <cstring>
#include <cstddef>

#ifndef MKL_LONG
#define MKL_LONG long
#endif

#include "mkl_dfti.h"

extern "C" {
/* mkl_free_buffers is not exported by libtorch_cpu.so; the reference only
 * calls it from FreeLibMem (src/JFFTMKLcore.cpp:78-81), so a no-op suffices. */
static inline void mkl_free_buffers(void) {}
/* Exported by libtorch_cpu.so; used by the reference-baseline driver to make
 * each worker thread run MKL sequentially (the reference links
 * mkl_sequential, JMultiSlice.h:27-29). */
int mkl_set_num_threads_local(int nt);
}

#ifndef _WIN32
/* Windows CRT bounds-checked memcpy: copies count bytes when they fit. */
static inline int memcpy_s(void* dst, size_t dstsz, const void* src, size_t count)
{
	if (dst == NULL || src == NULL) return 22;
	if (count > dstsz) { memset(dst, 0, dstsz); return 34; }
	memcpy(dst, src, count);
	return 0;
}
#endif
