// Gaussian reference weights of one atom and its species vectors, by one warp.
#pragma once

#include "d3_device.cuh"

namespace d3 {

constexpr double kWeightWf = 4.0;   // model.f90:80

// From the atom's CN: the Gaussian reference weights and their CN derivative
// with the reference's NaN/Inf fallback (weight_references,
// model.f90:201-324; FP64, lane r takes reference r, the sums run in
// reference order, so the weights equal those of a thread-per-atom loop bit
// for bit) and, when UV is given, the atom's species vectors
// UV[a][s] = U[a][s][0..7], dU[a][s][0..7] with U[a][s][r] =
// sum_q C6ref(r, q, s, s_a) gw_a[q] (the seven-term C6 dot products of the
// pair sweeps, get_atomic_c6, model.f90:432-461).
template <class R>
__device__ __forceinline__ void atom_weights(const Batch& b, const Species& s, const Config& c, const Work& w, int a,
                                             double cn, int lane, R* UV)
{
    const int sp = b.sp[a];
    const int nref = s.nref[sp];
    const double* cnref = s.refcn + sp * kMaxRef;
    const double wf2 = 2 * kWeightWf;
    const double cr = lane < nref ? cnref[lane] : 0.0;
    double g = 0.0;
    if (lane < nref) {
        const double d = cn - cr;
        g = exp(-kWeightWf * d * d);
    }
    double norm = 0.0, dnorm = 0.0, maxcn = cnref[0];
    for (int r = 0; r < nref; r++) {
        const double gr = __shfl_sync(0xffffffffu, g, r), crr = __shfl_sync(0xffffffffu, cr, r);
        norm = norm + gr;
        dnorm = dnorm + wf2 * (crr - cn) * gr;
        maxcn = fmax(maxcn, crr);
    }
    norm = 1.0 / norm;
    double gwk = 0.0, dgwk = 0.0;
    if (lane < nref) {
        const double expd = wf2 * (cr - cn) * g;
        gwk = g * norm;
        if (isnan(gwk) || isinf(gwk)) gwk = (maxcn == cr) ? 1.0 : 0.0;
        dgwk = expd * norm - g * dnorm * (norm * norm);
        if (isnan(dgwk) || isinf(dgwk)) dgwk = 0.0;
    }
    if (lane < kMaxRef) {
        w.gw[a * kMaxRef + lane] = gwk;
        w.dgw[a * kMaxRef + lane] = dgwk;
        if (c.mixed) {
            w.gwf[a * kMaxRef + lane] = float(gwk);
            w.dgwf[a * kMaxRef + lane] = float(dgwk);
        }
    }
    if (!UV) return;
    double gq[kMaxRef], dq[kMaxRef];
#pragma unroll
    for (int q = 0; q < kMaxRef; q++) {
        gq[q] = __shfl_sync(0xffffffffu, gwk, q);
        dq[q] = __shfl_sync(0xffffffffu, dgwk, q);
    }
    const bool ghost = b.ghost && b.ghost[a];
    const int nid = b.nid;
    R* o = UV + (size_t)a * nid * (2 * kRefPad);
    for (int e = lane; e < nid * kRefPad; e += 32) {
        const int sx = e / kRefPad, r = e % kRefPad;
        double u = 0.0, du = 0.0;
        if (!ghost && r < s.nref[sx]) {
            const double* ref = s.c6ref + ((size_t)(sx * nid + sp) * kMaxRef + r) * kMaxRef;
#pragma unroll
            for (int q = 0; q < kMaxRef; q++)
                if (q < nref) {
                    u += gq[q] * __ldg(ref + q);
                    du += dq[q] * __ldg(ref + q);
                }
        }
        o[sx * (2 * kRefPad) + r] = R(u);
        o[sx * (2 * kRefPad) + kRefPad + r] = R(du);
    }
}

}  // namespace d3
