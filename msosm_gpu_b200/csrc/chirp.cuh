// chirp.cuh -- the dedispersion chirp of the reference filter design on the
// device (msosm_prepare.cpp:50-62), shared by the block and large designs.
#pragma once

#include <cuda_runtime.h>

#include "host_prepare.hpp"

namespace msosm {

// Chirp phase at offset index i with the reference's rounding sequence
// (msosm_prepare.cpp:50-62): float w, float (w + w0), the rest in double,
// left to right.  Explicit round-to-nearest intrinsics keep the compiler
// from contracting any step into an FMA.
__device__ __forceinline__ double chirp_phase(const ChirpParams &p, unsigned int i)
{
    const double pi = kPi;
    const double fs = (double)p.fs;
    const float si = __fmul_rn(p.step, __uint2float_rn(i));
    float w = __double2float_rn(__dadd_rn(__dmul_rn(-pi, fs), (double)si));
    w = __double2float_rn(__dadd_rn((double)w, __dmul_rn(pi, fs)));
    const float den = __fadd_rn(w, p.w0);
    double ph = __dmul_rn(4.0, pi);
    ph = __dmul_rn(ph, pi);
    ph = __dmul_rn(ph, (double)p.kdm);
    ph = __dmul_rn(ph, (double)p.dm);
    ph = __dmul_rn(ph, (double)w);
    ph = __dmul_rn(ph, (double)w);
    ph = __ddiv_rn(ph, (double)den);
    ph = __ddiv_rn(ph, (double)p.w0);
    ph = __ddiv_rn(ph, (double)p.w0);
    return ph;
}

// cos/sin of a phase of up to ~1e7 rad: reduce mod 2 pi in FP64 with 2 pi
// split into a double head and tail (Cody-Waite), then sincos.
__device__ __forceinline__ void chirp_cis(double ph, float &c, float &s)
{
    constexpr double kTwoPiHi = 6.283185307179586232;     // nearest double to 2 pi
    constexpr double kTwoPiLo = 2.4492935982947064e-16;   // 2 pi - kTwoPiHi
    constexpr double kInvTwoPi = 0.15915494309189533577;
    const double n = rint(ph * kInvTwoPi);
    double r = fma(-n, kTwoPiHi, ph);
    r = fma(-n, kTwoPiLo, r);
    double sd, cd;
    sincos(r, &sd, &cd);
    c = (float)cd;
    s = (float)sd;
}

}  // namespace msosm
