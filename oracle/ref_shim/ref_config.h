/*
 * ref_config.h -- force-included (-include) in front of the reference sources
 * when they are compiled as a test checker.  It takes the place of the
 * reference's Parameter.h (same include guard, so that file is skipped) and
 * selects the compile-time switches of Parameter.h:8-21 from -D flags:
 *   IPPI_REF_MRT / IPPI_REF_RR  -> MRT / RRLBM instead of SRTLBM (BGK + nets)
 *   IPPI_REF_PESKIN             -> Dirac_Delta (4x4 Peskin IB kernel)
 *   IPPI_REF_SINGLE             -> SINGLE (REAL = float)
 * D2Q9, DirectForce and SmagorinskyByHybrid stay on, as in the shipped file.
 */
#ifndef PARAMETER_H
#define PARAMETER_H
#include <cmath>
#include <iostream>
#include <vector>
#define D2Q9
#define DirectForce
#define SmagorinskyByHybrid
#if defined(IPPI_REF_MRT)
#define MRT
#elif defined(IPPI_REF_RR)
#define RRLBM
#else
#define SRTLBM
#endif
#ifdef IPPI_REF_PESKIN
#define Dirac_Delta
#endif
#ifdef IPPI_REF_SINGLE
#define SINGLE
typedef float REAL;
#else
typedef double REAL;
#endif
#endif
