// jms_sizes.h -- supported line lengths of the fused passes and their
// two-factor split N = A * B (A, B <= 32, radices 2, 3, 4, 5), with the
// launcher templates that jms_inst_*.cu instantiate.
#pragma once
#include "jms_kernels.h"

#define JMS_SIZES(X) \
	X(16, 4, 4) X(24, 4, 6) X(32, 4, 8) X(40, 5, 8) X(48, 6, 8) X(64, 8, 8) X(80, 8, 10) X(96, 8, 12) \
	X(120, 10, 12) X(128, 8, 16) X(160, 10, 16) X(192, 12, 16) X(240, 15, 16) X(256, 16, 16) \
	X(320, 16, 20) X(384, 16, 24) X(480, 20, 24) X(512, 16, 32) X(640, 20, 32) X(720, 24, 30) \
	X(768, 24, 32) X(960, 30, 32) X(1024, 32, 32)

namespace jms {
template <int A, int B> int row_blocks_t(int ny);
template <int A, int B> cudaError_t launch_entry_t(const PassArgs& p, cudaStream_t s);
template <int A, int B> cudaError_t launch_row_t(const PassArgs& p, cudaStream_t s);
template <int A, int B> cudaError_t launch_col_t(const PassArgs& p, cudaStream_t s);
template <int A, int B> cudaError_t launch_exit_t(const PassArgs& p, cudaStream_t s);
} // namespace jms
