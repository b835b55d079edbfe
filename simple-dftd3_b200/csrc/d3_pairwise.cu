// Pairwise decomposition of the dispersion energy (get_pairwise_dispersion_v2,
// disp.f90:403-457), in FP64: the additive (two-body) energy of every atom
// pair and the non-additive (ATM) energy distributed over the pairs of each
// triple, as the matrices energy2[i][j] and energy3[i][j] of every system
// (input atom order, systems one after the other).
//
//   k_pw_c6        C6 of every ordered atom pair of each system (sorted order)
//   k_pairwise2    one block per atom i: the lanes take the partners j and sum
//                  the pair over all lattice translations; every (i, j) entry
//                  is written once by its row, no atomics
//   k_pairwise3    one thread per pair (i, j <= i) in the triple loop order of
//                  atm.f90:829-950 (i >= j >= k, translations of j and k); a
//                  sixth of each triple energy goes to each ordered pair of
//                  the triple, summed per thread and added with FP64 atomics
#include <cfloat>
#include <cstdint>

#include "d3_device.cuh"
#include "d3_atm_common.cuh"

namespace d3 {

namespace {

constexpr int kPwThreads = 128;

__device__ __forceinline__ int system_of_offset(const long long* off, int nsys, long long t)
{
    int lo = 0, hi = nsys - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) / 2;
        if (off[mid] <= t) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// C6 of the ordered pair (r, c) of each system (get_atomic_c6,
// model.f90:340-431); ghost atoms give 0.
__global__ void k_pw_c6(Batch b, Species s, Work w, const long long* off, long long total, double* c6)
{
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= total) return;
    const int sys = system_of_offset(off, b.nsys, t);
    const int a0 = b.atom_off[sys], n = b.atom_off[sys + 1] - a0;
    const long long e = t - off[sys];
    const int r = a0 + (int)(e / n), c = a0 + (int)(e % n);
    double v = 0.0;
    if (!(b.ghost && (b.ghost[r] || b.ghost[c]))) {
        const int sr = b.sp[r], sc = b.sp[c];
        const double* ref = s.c6ref + (size_t)(sr * b.nid + sc) * kMaxRef * kMaxRef;
        for (int ir = 0; ir < s.nref[sr]; ir++) {
            double a = 0.0;
            for (int jr = 0; jr < s.nref[sc]; jr++) a += w.gw[c * kMaxRef + jr] * __ldg(ref + ir * kMaxRef + jr);
            v += w.gw[r * kMaxRef + ir] * a;
        }
    }
    c6[t] = v;
}

// edisp of one (i, j, T) term without the smooth cutoff: the energy
// expressions of rational.f90:623-705, zero.f90:662-755 and the pairwise
// routines of mzero, optimizedpower, cso and z.f90, with the pair constants
// of the engine's table (rrij, q1..q5) and, for Z damping, zc = R0 C6.
__device__ double pw_edisp(const Damp& d, const double* pr, double r2, double zc)
{
    const double rrij = pr[0];
    const double r4 = r2 * r2, r6 = r4 * r2, r8 = r6 * r2;
    switch (d.kind) {
    case kRational:
        return d.s6 / (r6 + pr[1]) + d.s8 * rrij / (r8 + pr[2]);
    case kZero: {
        const double r1 = sqrt(r2);
        const double t6 = pow(pr[1] / r1, d.alp), t8 = pow(pr[2] / r1, d.alp + 2.0);
        return d.s6 / (1.0 + 6.0 * t6) / r6 + d.s8 * rrij / (1.0 + 6.0 * t8) / r8;
    }
    case kMZero: {
        const double r1 = sqrt(r2);
        const double t6 = pow(r1 * pr[1] + pr[3], -d.alp), t8 = pow(r1 * pr[2] + pr[3], -(d.alp + 2.0));
        return d.s6 / (1.0 + 6.0 * t6) / r6 + d.s8 * rrij / (1.0 + 6.0 * t8) / r8;
    }
    case kOptimizedPower: {
        const double ib = pow(r2, -0.5 * d.bet);
        return d.s6 / (r6 + pr[1] * ib) + d.s8 * rrij / (r8 + pr[2] * ib);
    }
    case kCSO: {
        const double sf = 1.0 / (1.0 + exp(sqrt(r2) - pr[2]));
        return (d.s6 + d.a1 * sf) / (r6 + pr[1]);
    }
    default:
        return d.s6 / (r6 + zc) + d.s8 * rrij / (r8 + zc * rrij);
    }
}

__global__ void __launch_bounds__(kPwThreads) k_pairwise2(Batch b, Species s, Damp d, Config c, const long long* off,
                                                           const double* c6, double* e2)
{
    const int p = blockIdx.x;
    const int sys = b.sys_of_atom[p];
    const int a0 = b.atom_off[sys], a1 = b.atom_off[sys + 1], n = a1 - a0;
    const int t0 = b.img_off[kImgDisp2 * (b.nsys + 1) + sys], t1 = b.img_off[kImgDisp2 * (b.nsys + 1) + sys + 1];
    const double xp = b.x[p], yp = b.y[p], zp = b.z[p];
    const double cut2 = c.cut2 * c.cut2;
    const int sp = b.sp[p];
    const double* crow = c6 + off[sys] + (long long)(p - a0) * n;
    double* erow = e2 + off[sys] + (long long)b.local[p] * n;
    for (int q = a0 + threadIdx.x; q < a1; q += blockDim.x) {
        const double c6pq = crow[q - a0];
        double sum = 0.0;
        if (c6pq != 0.0) {
            const double* pr = s.pair + kPairSlots * (sp * b.nid + b.sp[q]);
            const double zc = d.kind == kZDamping ? d.a1 / double(b.zid[p] + b.zid[q]) * c6pq : 0.0;
            const double dx = xp - b.x[q], dy = yp - b.y[q], dz = zp - b.z[q];
            for (int t = t0; t < t1; t++) {
                const double vx = dx - b.img[3 * t], vy = dy - b.img[3 * t + 1], vz = dz - b.img[3 * t + 2];
                const double r2 = vx * vx + vy * vy + vz * vz;
                if (r2 > cut2 || r2 < DBL_EPSILON) continue;
                double sw = 1.0, dsw = 0.0;
                if (c.width2 > 0.0) smooth<double>(sqrt(r2), c.cut2, c.width2, sw, dsw);
                sum -= 0.5 * c6pq * sw * pw_edisp(d, pr, r2, zc);
            }
        }
        erow[b.local[q]] = sum;
    }
}

__device__ __forceinline__ double pw_triple_scale(int i, int j, int k)
{
    // atm.f90:954-980
    if (i == j) return i == k ? 1.0 / 6.0 : 0.5;
    return (i != k && j != k) ? 1.0 : 0.5;
}

__global__ void __launch_bounds__(kPwThreads) k_pairwise3(Batch b, Species s, Damp d, Config c, const long long* off,
                                                           long long total, const double* c6, double* e3)
{
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= total) return;
    const int sys = system_of_offset(off, b.nsys, t);
    const int a0 = b.atom_off[sys], n = b.atom_off[sys + 1] - a0;
    const long long e = t - off[sys];
    const int pl = (int)(e / n), ql = (int)(e % n);
    if (ql > pl) return;                     // pairs (i, j <= i) only
    const int p = a0 + pl, q = a0 + ql;
    const double* cm = c6 + off[sys];
    const double c6pq = cm[(long long)pl * n + ql];
    if (c6pq == 0.0) return;
    const int t0 = b.img_off[kImgDisp3 * (b.nsys + 1) + sys], t1 = b.img_off[kImgDisp3 * (b.nsys + 1) + sys + 1];
    const double cut2 = c.cut3 * c.cut3;
    const bool smooth_on = c.width3 > 0.0;
    const double alp3 = (d.alp + 2.0) / 3.0;
    const int sp = b.sp[p], sq = b.sp[q];
    const double r0pq = s.atm_r0[sp * b.nid + sq];     // rs9 R0 (rs9 = 4/3)
    const double xp = b.x[p], yp = b.y[p], zp = b.z[p];
    double* eg = e3 + off[sys];
    const long long lp = b.local[p], lq = b.local[q];
    double epq = 0.0;
    for (int tj = t0; tj < t1; tj++) {
        const double ijx = b.x[q] + b.img[3 * tj] - xp, ijy = b.y[q] + b.img[3 * tj + 1] - yp,
                     ijz = b.z[q] + b.img[3 * tj + 2] - zp;
        const double r2ij = ijx * ijx + ijy * ijy + ijz * ijz;
        if (r2ij > cut2 || r2ij < DBL_EPSILON) continue;
        double swij = 1.0, dsw = 0.0;
        if (smooth_on) smooth<double>(sqrt(r2ij), c.cut3, c.width3, swij, dsw);
        for (int rl = 0; rl <= ql; rl++) {
            const int r = a0 + rl;
            const double c6pr = cm[(long long)pl * n + rl], c6qr = cm[(long long)ql * n + rl];
            const double c9 = -d.s9 * sqrt(fabs(c6pq * c6pr * c6qr));
            if (c9 == 0.0) continue;
            const int sr = b.sp[r];
            const double r0 = r0pq * s.atm_r0[sp * b.nid + sr] * s.atm_r0[sq * b.nid + sr];
            const double triple = pw_triple_scale(pl, ql, rl);
            double epr = 0.0, eqr = 0.0;
            for (int tk = t0; tk < t1; tk++) {
                const double ikx = b.x[r] + b.img[3 * tk] - xp, iky = b.y[r] + b.img[3 * tk + 1] - yp,
                             ikz = b.z[r] + b.img[3 * tk + 2] - zp;
                const double r2ik = ikx * ikx + iky * iky + ikz * ikz;
                if (r2ik > cut2 || r2ik < DBL_EPSILON) continue;
                const double jkx = ikx - ijx, jky = iky - ijy, jkz = ikz - ijz;
                const double r2jk = jkx * jkx + jky * jky + jkz * jkz;
                if (r2jk > cut2 || r2jk < DBL_EPSILON) continue;
                double sw = swij;
                if (smooth_on) {
                    double swik, swjk;
                    smooth<double>(sqrt(r2ik), c.cut3, c.width3, swik, dsw);
                    smooth<double>(sqrt(r2jk), c.cut3, c.width3, swjk, dsw);
                    sw *= swik * swjk;
                }
                const double r2 = r2ij * r2ik * r2jk;
                const double r1 = sqrt(r2), r3 = r2 * r1, r5 = r3 * r2;
                const double fdmp = 1.0 / (1.0 + 6.0 * pow(r0 / r1, alp3));
                const double ang = 0.375 * (r2ij + r2jk - r2ik) * (r2ij - r2jk + r2ik) * (-r2ij + r2jk + r2ik) / r5
                                 + 1.0 / r3;
                const double de = ang * fdmp * c9 * triple * sw / 6.0;
                epq -= de;
                epr -= de;
                eqr -= de;
            }
            if (epr != 0.0) {
                const long long lr = b.local[r];
                atomicAdd(eg + lp * n + lr, epr);
                atomicAdd(eg + lr * n + lp, epr);
                atomicAdd(eg + lq * n + lr, eqr);
                atomicAdd(eg + lr * n + lq, eqr);
            }
        }
    }
    if (epq != 0.0) {
        atomicAdd(eg + lp * n + lq, epq);
        atomicAdd(eg + lq * n + lp, epq);
    }
}

}  // namespace

void launch_pairwise(const Batch& b, const Species& s, const Damp& d, const Config& c, const Work& w,
                     const long long* off, long long total, double* c6, double* e2, double* e3,
                     cudaStream_t stream)
{
    if (b.natoms <= 0 || total <= 0) return;
    const unsigned blocks = (unsigned)((total + kPwThreads - 1) / kPwThreads);
    k_pw_c6<<<blocks, kPwThreads, 0, stream>>>(b, s, w, off, total, c6);
    k_pairwise2<<<b.natoms, kPwThreads, 0, stream>>>(b, s, d, c, off, c6, e2);
    cudaMemsetAsync(e3, 0, sizeof(double) * total, stream);
    if (std::fabs(d.s9) >= DBL_EPSILON)
        k_pairwise3<<<blocks, kPwThreads, 0, stream>>>(b, s, d, c, off, total, c6, e3);
}

}  // namespace d3
