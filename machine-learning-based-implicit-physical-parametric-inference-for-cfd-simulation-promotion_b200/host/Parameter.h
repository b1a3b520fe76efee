// Parameter.h -- compile-time switches of the host driver, the same macro
// names as the reference's IPPI-LBM/Parameter.h, mapped onto ippi_params.
//
//   collision   SRTLBM (default) | MRT | RRLBM
//   SINGLE      FP32 populations and arithmetic (REAL = float); otherwise FP64
//   HALF_STORAGE / BF16_STORAGE   FP16 / BF16 population storage, FP32
//               arithmetic (no counterpart in the reference)
//   Dirac_Delta 4-point Peskin immersed-boundary kernel; otherwise bilinear
//   SmagorinskyByHybrid  Smagorinsky relaxation time (on unless NO_LES)
//
// Velocity set, in the order every population array uses (NodeAndLattice.cpp
// e[9][2]):
//   k   0  1  2  3  4  5  6  7  8
//   x   0 +1  0 -1  0 +1 -1 -1 +1
//   y   0  0 +1  0 -1 +1 +1 -1 -1
#ifndef PARAMETER_H
#define PARAMETER_H
#include <cmath>
#include <iostream>
#include <vector>

#include "ippi_lbm.h"

#ifndef D2Q9
#define D2Q9
#endif
#define DirectForce
#if !defined(SRTLBM) && !defined(MRT) && !defined(RRLBM)
#define SRTLBM
#endif
#if !defined(NO_LES) && !defined(SmagorinskyByHybrid)
#define SmagorinskyByHybrid
#endif

#ifdef SINGLE
typedef float REAL;
#else
typedef double REAL;
#endif

namespace ippi_host {
#if defined(MRT)
constexpr int kCollision = IPPI_MRT;
#elif defined(RRLBM)
constexpr int kCollision = IPPI_RR;
#else
constexpr int kCollision = IPPI_BGK;
#endif
#if defined(HALF_STORAGE)
constexpr int kStorage = IPPI_F16;
#elif defined(BF16_STORAGE)
constexpr int kStorage = IPPI_BF16;
#elif defined(SINGLE)
constexpr int kStorage = IPPI_F32;
#else
constexpr int kStorage = IPPI_F64;
#endif
#ifdef Dirac_Delta
constexpr int kDelta = IPPI_DELTA_PESKIN4;
#else
constexpr int kDelta = IPPI_DELTA_BILINEAR;
#endif
#ifdef SmagorinskyByHybrid
constexpr int kLes = IPPI_LES_SMAGORINSKY;
#else
constexpr int kLes = IPPI_LES_NONE;
#endif
}  // namespace ippi_host

#endif
