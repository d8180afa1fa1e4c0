// jms_sizes.h -- supported line lengths and the candidate line plans of each
// (jms_passes.cuh).  Plan<A, B, C> splits N = A * B (A, B <= 32, radices 2, 3,
// 4, 5; paired threads when B = 2A); Plan3<R, C> runs N = R^3 in three stages;
// C is the column-pass tile width.  The first plan of a length is its default;
// JMS_Autotune picks among the candidates by timing them (jms_tune.cpp).
#pragma once
#include "jms_kernels.h"

namespace jms {
template <int A, int B, int CC = 16> struct Plan;
template <int R, int CC> struct Plan3;

using P16 = Plan<4, 4, 16>;
using P24 = Plan<4, 6, 16>;
using P32 = Plan<4, 8, 16>;
using P40 = Plan<5, 8, 16>;
using P48 = Plan<6, 8, 16>;
using P64a = Plan<8, 8, 16>;
using P64b = Plan3<4, 16>;
using P80 = Plan<8, 10, 16>;
using P96 = Plan<8, 12, 16>;
using P120 = Plan<10, 12, 16>;
using P128a = Plan<8, 16, 16>;
using P128b = Plan<16, 8, 16>;
using P160 = Plan<10, 16, 16>;
using P180 = Plan<12, 15, 16>;
using P192 = Plan<12, 16, 16>;
using P240 = Plan<15, 16, 16>;
using P256a = Plan<16, 16, 16>;
using P256b = Plan<16, 16, 8>;
using P320 = Plan<16, 20, 16>;
using P384 = Plan<16, 24, 16>;
using P480 = Plan<20, 24, 16>;
using P512a = Plan<16, 32, 16>;
using P512b = Plan3<8, 8>;
using P512c = Plan<16, 32, 8>;
using P640 = Plan<20, 32, 16>;
using P720 = Plan<24, 30, 16>;
using P768 = Plan<24, 32, 16>;
using P960 = Plan<30, 32, 16>;
using P1024a = Plan<32, 32, 16>;
using P1024b = Plan<32, 32, 8>;
using P2048a = Plan<32, 64, 8>;
using P2048b = Plan<32, 64, 4>;

template <class PL> int row_blocks_t(int ny);
template <class PL> cudaError_t launch_entry_t(const PassArgs& p, cudaStream_t s);
template <class PL> cudaError_t launch_row_t(const PassArgs& p, cudaStream_t s);
template <class PL> cudaError_t launch_col_t(const PassArgs& p, cudaStream_t s);
template <class PL> cudaError_t launch_exit_t(const PassArgs& p, cudaStream_t s);
} // namespace jms

// X(length, plan alias, printable name); the first entry of a length is its default
#define JMS_PLANS(X) \
	X(16, P16, "4x16") X(24, P24, "4x6") X(32, P32, "4x8 pair") X(40, P40, "5x8") X(48, P48, "6x8") \
	X(64, P64a, "8x8") X(64, P64b, "4x4x4") X(80, P80, "8x10") X(96, P96, "8x12") X(120, P120, "10x12") \
	X(128, P128a, "8x16 pair") X(128, P128b, "16x8") X(160, P160, "10x16") X(180, P180, "12x15") X(192, P192, "12x16") \
	X(240, P240, "15x16") X(256, P256a, "16x16 c16") X(256, P256b, "16x16 c8") X(320, P320, "16x20") \
	X(384, P384, "16x24") X(480, P480, "20x24") X(512, P512a, "16x32 pair c16") X(512, P512b, "8x8x8 c8") \
	X(512, P512c, "16x32 pair c8") \
	X(640, P640, "20x32") X(720, P720, "24x30") X(768, P768, "24x32") \
	X(960, P960, "30x32") X(1024, P1024a, "32x32 c16") X(1024, P1024b, "32x32 c8") \
	X(2048, P2048a, "32x64 pair c8") X(2048, P2048b, "32x64 pair c4")

// X(length, plan alias): the default (first) plan of every length in
// JMS_PLANS, in three groups (used by the phase-grating generator,
// jms_pgr_ops_*.cu)
#define JMS_DEFAULT_PLANS_0(X) \
	X(16, P16) X(24, P24) X(32, P32) X(40, P40) X(48, P48) X(64, P64a) X(80, P80) X(96, P96) X(120, P120) \
	X(128, P128a) X(160, P160) X(180, P180) X(192, P192) X(240, P240) X(256, P256a)
#define JMS_DEFAULT_PLANS_1(X) X(320, P320) X(384, P384) X(480, P480) X(512, P512a) X(640, P640) X(720, P720)
#define JMS_DEFAULT_PLANS_2(X) X(768, P768) X(960, P960) X(1024, P1024a) X(2048, P2048a)
