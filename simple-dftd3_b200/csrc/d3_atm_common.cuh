// Per-triple arithmetic shared by the ATM kernels (d3_atm.cu: neighbour-list
// roots, d3_atm_mol.cu: molecules per block).
#pragma once

#include <cfloat>

#include "d3_device.cuh"

namespace d3 {
namespace {

// {sqrt(C6_rc), dC6_rc/dCN_r / C6_rc, dC6_rc/dCN_c / C6_rc} of an ordered atom
// pair (r, c) of a system (get_atomic_c6, model.f90:432-461), ghosts giving 0,
// and alp3 log(r0_rc) of the ATM damping radius (atm.f90:744-749; natural log
// in the FP64 form, base 2 in the mixed form).  One aligned vector load.
template <class R>
struct __align__(4 * sizeof(R)) C6Entry { R sc6, qrc, qcr, lr0; };

template <class R>
__device__ __forceinline__ R rsqrt_r(R x) { if constexpr (sizeof(R) == 8) return rsqrt(x); else return rsqrtf(x); }

// Reciprocal of the triple arithmetic: IEEE in the FP64 form, the hardware
// approximation (a few ulp) in the FP32 part of the mixed form.
template <class R>
__device__ __forceinline__ R rcp_r(R x) { if constexpr (sizeof(R) == 8) return R(1) / x; else return __fdividef(1.0f, x); }

// log and exp in the precision of the form (natural base for FP64, base 2
// with the hardware units for FP32; only their composition matters).
template <class R>
__device__ __forceinline__ R rlog(R x) { if constexpr (sizeof(R) == 8) return log(x); else return __log2f(x); }
template <class R>
__device__ __forceinline__ R rexp(R x) { if constexpr (sizeof(R) == 8) return exp(x); else return exp2f(x); }

template <class R>
__device__ __forceinline__ void smooth(R r, R cutoff, R width, R& sw, R& dsw)
{
    // cutoff.f90:73-99
    if (width <= R(0) || width >= cutoff) { sw = R(1); dsw = R(0); return; }
    const R inner = cutoff - width;
    if (r <= inner) { sw = R(1); dsw = R(0); }
    else if (r >= cutoff) { sw = R(0); dsw = R(0); }
    else {
        const R x = (cutoff - r) / width;
        sw = x * x * x * (R(10) + x * (R(-15) + R(6) * x));
        dsw = R(-30) * x * x * (R(1) - x) * (R(1) - x) / width;
    }
}

__device__ __forceinline__ bool owns_pair_atm(const Partition& p, int i, int j)
{
    long long hi = i > j ? i : j, lo = i > j ? j : i;
    return (hi * (hi + 1) / 2 + lo) % p.nparts == p.part;
}

// P(x; y, z) = x^3 + x^2 (y + z) + x (3 y^2 + 2 y z + 3 z^2) - 5 (y - z)^2 (y + z),
// the numerator of the angular derivative along x (atm.f90:751-776), with
// s1 = x + y + z.
template <class R>
__device__ __forceinline__ R ang_deriv(R x, R y, R z, R s1)
{
    const R u = y + z, d = y - z;
    const R w = d * d;
    return x * (x * s1 + w + R(2) * u * u) - R(5) * u * w;
}

}  // namespace
}  // namespace d3
