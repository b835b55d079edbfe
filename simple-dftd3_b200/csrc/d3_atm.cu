// Axilrod-Teller-Muto three-body dispersion (get_atm_dispersion, atm.f90:433-825)
// with energy, gradient, virial and dE/dCN.
//
// Enumeration: every atom i (the root) owns the triples whose other two
// members are neighbours (j, T_j), (k, T_k) within the three-body cutoff with
// k <= j <= i in the batch atom order -- the reference's i >= j >= k loop
// (atm.f90:705-733) over any fixed atom order, so every triple is counted once
// and triple_scale (atm.f90:954-980) handles repeated atoms.
//
// Pipeline:
//   k_c6_matrix     dense per-system table {sqrt(C6), dC6_rc/dCN_r / C6,
//                   dC6_rc/dCN_c / C6} for the (j, k) lookups of the triples
//   k_nbr_count     neighbour entries (j <= i, T) of every root
//   (device scan)   entry offsets
//   k_nbr_fill      entries sorted by j, then T: vector x_j + T - x_i, r^2 and
//                   the end of the entry's atom group
//   k_triples       persistent blocks take roots from a queue (largest lists
//                   first); a 16 x 16 thread grid sweeps 32 x 64 tiles of
//                   (j-entry, k-entry) pairs, 2 x 4 per thread, with register
//                   accumulators per entry.  Per-entry sums (scalar pair factor
//                   S, energy D, jk-gradient G, jk-dC6 term Q) are reduced
//                   within the block in a fixed order and scattered once per
//                   entry (FP64 atomics into the gradient and dE/dCN of the
//                   partner atoms).
#include <cub/cub.cuh>

#include <algorithm>

#include <cfloat>
#include <cstdint>

#include "d3_device.cuh"
#include "d3_atm_common.cuh"

namespace d3 {

namespace {

constexpr int kTA = 32;          // j-entries per tile
constexpr int kTB = 64;          // k-entries per tile
constexpr int kThreadsAtm = 256; // 16 x 16
constexpr int kAcc = 5;          // per-entry accumulators: S, Gx, Gy, Gz, dE/dCN of the partner

// ------------------------------------------------------------ C6 matrix ----

// {sqrt(C6_rc), dC6_rc/dCN_r / C6_rc, dC6_rc/dCN_c / C6_rc} for every ordered
// pair (r, c) of each system (get_atomic_c6, model.f90:432-461); ghosts give 0.
template <class R>
__global__ void k_c6_matrix(Batch b, Species s, Work w, double alp3, const long long* mat_off, C6Entry<R>* mat,
                            long long total)
{
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= total) return;
    // locate the system by binary search over the matrix offsets
    int lo = 0, hi = b.nsys - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) / 2;
        if (mat_off[mid] <= t) lo = mid; else hi = mid - 1;
    }
    const int sys = lo;
    const int a0 = b.atom_off[sys];
    const int n = b.atom_off[sys + 1] - a0;
    const long long e = t - mat_off[sys];
    const int r = a0 + (int)(e / n), c = a0 + (int)(e % n);
    const double r0 = __ldg(s.atm_r0 + b.sp[r] * b.nid + b.sp[c]);
    const R lr0 = R(alp3 * (sizeof(R) == 8 ? log(r0) : log2(r0)));
    C6Entry<R> out{R(0), R(0), R(0), lr0};
    const bool ghost = b.ghost && (b.ghost[r] || b.ghost[c]);
    if (!ghost) {
        const int sr = b.sp[r], sc = b.sp[c];
        const int nr = s.nref[sr], nc = s.nref[sc];
        const double* ref = s.c6ref + (size_t)(sr * b.nid + sc) * kMaxRef * kMaxRef;
        double c6 = 0.0, dr = 0.0, dc = 0.0;
        for (int ir = 0; ir < nr; ir++) {
            double a = 0.0, bb = 0.0;
            for (int jr = 0; jr < nc; jr++) {
                const double v = __ldg(ref + ir * kMaxRef + jr);
                a += w.gw[c * kMaxRef + jr] * v;
                bb += w.dgw[c * kMaxRef + jr] * v;
            }
            c6 += w.gw[r * kMaxRef + ir] * a;
            dr += w.dgw[r * kMaxRef + ir] * a;
            dc += w.gw[r * kMaxRef + ir] * bb;
        }
        if (c6 != 0.0) out = C6Entry<R>{R(sqrt(c6)), R(dr / c6), R(dc / c6), lr0};
    }
    mat[t] = out;
}

// --------------------------------------------------------- neighbour lists --

__device__ __forceinline__ bool in_shell(double r2, double cut2) { return !(r2 > cut2 || r2 < DBL_EPSILON); }

// Number of entries (j <= i, T) with eps <= |x_j + T - x_i|^2 <= cutoff^2.
__global__ void k_nbr_count(Batch b, Config c, const uint8_t* sys_skip, int* cnt, int* max_cnt)
{
    const int lane = threadIdx.x & 31;
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (i >= b.natoms) return;
    const int sys = b.sys_of_atom[i];
    if (sys_skip && sys_skip[sys]) {
        if (lane == 0) cnt[i] = 0;
        return;
    }
    const int j0 = b.atom_off[sys];
    const int t0 = b.img_off[kImgDisp3 * (b.nsys + 1) + sys], t1 = b.img_off[kImgDisp3 * (b.nsys + 1) + sys + 1];
    const double xi = b.x[i], yi = b.y[i], zi = b.z[i];
    const double cut2 = c.cut3 * c.cut3;
    int n = 0;
    for (int j = j0 + lane; j <= i; j += 32) {
        const double dx = b.x[j] - xi, dy = b.y[j] - yi, dz = b.z[j] - zi;
        for (int t = t0; t < t1; t++) {
            const double vx = dx + __ldg(b.img + 3 * t), vy = dy + __ldg(b.img + 3 * t + 1),
                         vz = dz + __ldg(b.img + 3 * t + 2);
            n += in_shell(vx * vx + vy * vy + vz * vz, cut2);
        }
    }
    for (int off = 16; off > 0; off >>= 1) n += __shfl_xor_sync(0xffffffffu, n, off);
    if (lane == 0) {
        cnt[i] = n;
        atomicMax(max_cnt, n);
    }
}

__global__ void k_atm_guard(const long long* total, const int* max_cnt, long long cap, int stride, int* guard)
{
    *guard = (*total > cap || *max_cnt > stride) ? 1 : 0;
}

// Entries of root i in (j, T) order.  vec = (x_j + T) - x_i as in atm.f90:718.
__global__ void k_nbr_fill(Batch b, Config c, const uint8_t* sys_skip, const long long* off, int* nbr_j,
                           int* nbr_gend, double4* nbr_v, const int* guard)
{
    const int lane = threadIdx.x & 31;
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (i >= b.natoms || *guard) return;
    const int sys = b.sys_of_atom[i];
    if (sys_skip && sys_skip[sys]) return;   // no entries were counted for this root
    const int j0 = b.atom_off[sys];
    const int t0 = b.img_off[kImgDisp3 * (b.nsys + 1) + sys], t1 = b.img_off[kImgDisp3 * (b.nsys + 1) + sys + 1];
    const double xi = b.x[i], yi = b.y[i], zi = b.z[i];
    const double cut2 = c.cut3 * c.cut3;
    long long pos = off[i];
    for (int jb = j0; jb <= i; jb += 32) {
        const int j = jb + lane;
        const bool valid = j <= i;
        const double dx = valid ? b.x[j] - xi : 0.0, dy = valid ? b.y[j] - yi : 0.0, dz = valid ? b.z[j] - zi : 0.0;
        int n = 0;
        if (valid)
            for (int t = t0; t < t1; t++) {
                const double vx = dx + __ldg(b.img + 3 * t), vy = dy + __ldg(b.img + 3 * t + 1),
                             vz = dz + __ldg(b.img + 3 * t + 2);
                n += in_shell(vx * vx + vy * vy + vz * vz, cut2);
            }
        // exclusive prefix over the lanes keeps the entries sorted by j
        int incl = n;
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        const int total = __shfl_sync(0xffffffffu, incl, 31);
        long long p = pos + incl - n;
        const int gend = (int)(pos - off[i]) + incl;   // group end, local to the root's list
        if (valid && n > 0)
            for (int t = t0; t < t1; t++) {
                const double vx = dx + __ldg(b.img + 3 * t), vy = dy + __ldg(b.img + 3 * t + 1),
                             vz = dz + __ldg(b.img + 3 * t + 2);
                const double r2 = vx * vx + vy * vy + vz * vz;
                if (!in_shell(r2, cut2)) continue;
                nbr_j[p] = j;
                nbr_gend[p] = gend;
                nbr_v[p] = make_double4(vx, vy, vz, r2);
                p++;
            }
        pos += total;
    }
}

// ------------------------------------------------------------ triple sum ----

template <class R> struct Vec4;
template <> struct Vec4<double> { using type = double4; };
template <> struct Vec4<float> { using type = float4; };

// One neighbour entry of the current root, precomputed once per root.
template <class R>
struct Slot {
    typename Vec4<R>::type v;   // head of x_j + T - x_i, r^2
    typename Vec4<R>::type l;   // tail of the vector (mixed form), 1/r^2
    typename Vec4<R>::type c;   // sqrt(C6_ij), dC6_ij/dCN_i / C6, dC6_ij/dCN_j / C6, alp3 log(r0_ij / r_ij)
    typename Vec4<R>::type s;   // 1/r, switch, dsw/dr / r, -
    int4 meta;                  // atom, group end, species, input index
};

template <class R, bool GRAD, bool PER>
__global__ void __launch_bounds__(kThreadsAtm, sizeof(R) == 4 ? 3 : 1) k_triples(Batch b, Species sp, Damp d, Config c, Partition part,
                                                         Work w, const C6Entry<R>* mat, const long long* mat_off,
                                                         const long long* off, const int* cnt, const int* nbr_j,
                                                         const int* nbr_gend, const double4* nbr_v,
                                                         unsigned int* queue, double* slot_acc, Slot<R>* slot_scr,
                                                         int slot_stride, double* e3, double* sig3)
{
    // dynamic shared memory: entry tiles, C6 of the tile's (j, k) pairs, k-role reduction
    extern __shared__ __align__(16) unsigned char smem[];
    Slot<R>* sa = reinterpret_cast<Slot<R>*>(smem);
    Slot<R>* sb = sa + kTA;
    auto sjk = reinterpret_cast<C6Entry<R>(*)[kTB]>(sb + kTB);
    auto kred = reinterpret_cast<R(*)[kTB / 2][kAcc]>(sjk + kTA);
    __shared__ int s_root;
    __shared__ double wsum[kThreadsAtm / 32][13];
    const int tid = threadIdx.x;
    const int tx = tid & 15, ty = tid >> 4;
    const int lane = tid & 31;
    double* acc = slot_acc + (size_t)blockIdx.x * slot_stride * kAcc;
    Slot<R>* scr = slot_scr + (size_t)blockIdx.x * slot_stride;
    const R s9 = R(d.s9);
    const R alp = R(d.alp + 2.0);        // ATM exponent alp + 2 (rational.f90:563)
    const R alp3 = alp / R(3);
    const R cut2 = R(c.cut3 * c.cut3);
    const bool smooth_on = c.width3 > 0.0 && c.width3 < c.cut3;
    const R cutoff = R(c.cut3), width = R(c.width3);
    if (w.atm_guard && *w.atm_guard) return;   // lists did not fit the reserved buffers
    __syncthreads();

    for (;;) {
        if (tid == 0) {
            const unsigned q = atomicAdd(queue, 1u);
            s_root = q < (unsigned)b.natoms ? b.natoms - 1 - (int)q : -1;
        }
        __syncthreads();
        const int i = s_root;
        __syncthreads();
        if (i < 0) break;
        const int m = cnt[i];
        const long long base = off[i];
        const int sys = b.sys_of_atom[i];
        const int a0 = b.atom_off[sys];
        const int nsys_n = b.atom_off[sys + 1] - a0;
        const long long mbase = mat_off[sys];
        const long long mrow_i = mbase + (long long)(i - a0) * nsys_n;
        const int orig_i = b.local[i];
        const int si = b.sp[i];
        double e_root = 0.0, dei = 0.0;
        double sxx = 0, syy = 0, szz = 0, sxy = 0, sxz = 0, syz = 0;
        int ntrip = 0;
        if (m > 0) {
            // entry records of this root (all threads)
            for (int k = tid; k < m; k += kThreadsAtm) {
                const int j = nbr_j[base + k];
                const double4 v = nbr_v[base + k];
                Slot<R> r;
                const int sj = b.sp[j];
                const C6Entry<R> e = mat[mrow_i + (j - a0)];
                const double r0 = __ldg(sp.atm_r0 + si * b.nid + sj);
                if constexpr (sizeof(R) == 8) {
                    r.v = make_double4(v.x, v.y, v.z, v.w);
                    r.l = make_double4(0.0, 0.0, 0.0, 1.0 / v.w);
                    const double rs = rsqrt(v.w);
                    r.c = make_double4(e.sc6, e.qrc, e.qcr, alp3 * (log(r0) - 0.5 * log(v.w)));
                    r.s = make_double4(rs, 1.0, 0.0, 0.0);
                } else {
                    const float hx = __double2float_rn(v.x), hy = __double2float_rn(v.y), hz = __double2float_rn(v.z);
                    r.v = make_float4(hx, hy, hz, __double2float_rn(v.w));
                    r.l = make_float4(__double2float_rn(v.x - (double)hx), __double2float_rn(v.y - (double)hy),
                                      __double2float_rn(v.z - (double)hz), __double2float_rn(1.0 / v.w));
                    r.c = make_float4(e.sc6, e.qrc, e.qcr,
                                      __double2float_rn(double(alp3) * (log2(r0) - 0.5 * log2(v.w))));
                    r.s = make_float4(__double2float_rn(rsqrt(v.w)), 1.f, 0.f, 0.f);
                }
                if (smooth_on) {
                    R sw, dsw;
                    const R rr = R(sqrt(v.w));
                    smooth<R>(rr, cutoff, width, sw, dsw);
                    r.s.y = sw;
                    r.s.z = dsw / rr;
                }
                r.meta = make_int4(j, nbr_gend[base + k], sj, b.local[j]);
                scr[k] = r;
                if (GRAD)
                    for (int v2 = 0; v2 < kAcc; v2++) acc[k * kAcc + v2] = 0.0;
            }
            __syncthreads();
            for (int B0 = 0; B0 < m; B0 += kTB) {
                __syncthreads();
                for (int k = tid; k < kTB; k += kThreadsAtm)
                    if (B0 + k < m) sb[k] = scr[B0 + k];
                __syncthreads();
                // first j-entry whose atom group reaches this k-tile
                int astart = B0;
                while (astart > 0 && sb[0].meta.x == scr[astart - 1].meta.x) astart--;
                R kacc[4][kAcc];
#pragma unroll
                for (int q = 0; q < 4; q++)
#pragma unroll
                    for (int v = 0; v < kAcc; v++) kacc[q][v] = R(0);
                for (int A0 = (astart / kTA) * kTA; A0 < m; A0 += kTA) {
                    __syncthreads();
                    for (int k = tid; k < kTA; k += kThreadsAtm)
                        if (A0 + k < m) sa[k] = scr[A0 + k];
                    __syncthreads();
                    // C6 table of the tile's (j, k) atom pairs
                    for (int k = tid; k < kTA * kTB; k += kThreadsAtm) {
                        const int ia = k / kTB, ib = k % kTB;
                        if (A0 + ia < m && B0 + ib < m && B0 + ib < sa[ia].meta.y)
                            sjk[ia][ib] = mat[mbase + (long long)(sa[ia].meta.x - a0) * nsys_n + (sb[ib].meta.x - a0)];
                    }
                    __syncthreads();
                    R jacc[2][kAcc];
#pragma unroll
                    for (int p = 0; p < 2; p++)
#pragma unroll
                        for (int v = 0; v < kAcc; v++) jacc[p][v] = R(0);
                    R te = R(0), tde = R(0), txx = R(0), tyy = R(0), tzz = R(0), txy = R(0), txz = R(0), tyz = R(0);
#pragma unroll
                    for (int p = 0; p < 2; p++) {
                        const int ia = ty + 16 * p;
                        if (A0 + ia >= m) continue;
                        const Slot<R>& A = sa[ia];
#pragma unroll
                        for (int q = 0; q < 4; q++) {
                            const int ib = tx + 16 * q;
                            const int kb = B0 + ib;
                            if (kb >= m || kb >= A.meta.y) continue;
                            const Slot<R>& Bs = sb[ib];
                            // j-k vector: (x_k + T_k - x_i) - (x_j + T_j - x_i)
                            R vx, vy, vz;
                            if constexpr (sizeof(R) == 8) {
                                vx = Bs.v.x - A.v.x; vy = Bs.v.y - A.v.y; vz = Bs.v.z - A.v.z;
                            } else {
                                vx = (Bs.v.x - A.v.x) + (Bs.l.x - A.l.x);
                                vy = (Bs.v.y - A.v.y) + (Bs.l.y - A.l.y);
                                vz = (Bs.v.z - A.v.z) + (Bs.l.z - A.l.z);
                            }
                            const R rc = vx * vx + vy * vy + vz * vz;   // r_jk^2
                            if (rc > cut2 || rc < R(DBL_EPSILON)) continue;
                            // a ghost gives C6 = 0 and with it zero contributions
                            const C6Entry<R> ejk = sjk[ia][ib];
                            if (part.nparts > 1) {
                                // owner of the triple: the pair of its two largest input indices
                                int o1 = orig_i, o2 = A.meta.w, o3 = Bs.meta.w, t;
                                if (o2 > o1) { t = o1; o1 = o2; o2 = t; }
                                if (o3 > o2) { t = o2; o2 = o3; o3 = t; }
                                if (o2 > o1) { t = o1; o1 = o2; o2 = t; }
                                if (!owns_pair_atm(part, o1, o2)) continue;
                            }
                            const R ra = A.v.w, rb = Bs.v.w;            // r_ij^2, r_ik^2
                            const R rsc = rsqrt_r<R>(rc);
                            const R irc = rsc * rsc;
                            const R ir1 = A.s.x * Bs.s.x * rsc;         // 1 / (r_ij r_ik r_jk)
                            const R ir2 = ir1 * ir1;
                            const R ir3 = ir2 * ir1;
                            const R ir5 = ir3 * ir2;

                            // (r0/r1)^alp3, r0 = r0ij r0ik r0jk, r1 = r_ij r_ik r_jk
                            const R t = rexp<R>(A.c.w + Bs.c.w + ejk.lr0 - R(0.5) * alp3 * rlog<R>(rc));
                            const R fdmp = rcp_r<R>(R(1) + R(6) * t);
                            const R s1 = ra + rb + rc;
                            const R ang = R(0.375) * (s1 - R(2) * rb) * (s1 - R(2) * rc) * (s1 - R(2) * ra) * ir5 + ir3;
                            const R c9 = -s9 * A.c.x * Bs.c.x * ejk.sc6;
                            const int jat = A.meta.x, kat = Bs.meta.x;
                            // triple_scale (atm.f90:954-980): repeated atoms only under periodicity
                            R triple = R(1);
                            if (PER) {
                                if (i == jat) triple = (i == kat) ? R(1.0 / 6.0) : R(0.5);
                                else triple = (i != kat && jat != kat) ? R(1) : R(0.5);
                            }
                            R sw = R(1), swjk = R(1), dswjkr = R(0);
                            if (smooth_on) {
                                R dsw;
                                const R rjk = rc * rsc;
                                smooth<R>(rjk, cutoff, width, swjk, dsw);
                                dswjkr = dsw * rsc;
                                sw = A.s.y * Bs.s.y * swjk;
                            }
                            const R dE0 = ang * fdmp * c9;
                            const R dE = dE0 * triple * sw;
                            te -= dE;
                            ntrip++;
                            if (!GRAD) continue;
                            // ds/dr2 pieces: common damping part and the angular parts
                            const R common = c9 * ang * (R(-2) * alp * t * (fdmp * fdmp));
                            const R kfac = R(0.375) * c9 * fdmp * ir5;
                            R sij = sw * (common + kfac * ang_deriv<R>(ra, rc, rb, s1)) * A.l.w;
                            R sik = sw * (common + kfac * ang_deriv<R>(rb, rc, ra, s1)) * Bs.l.w;
                            R sjk = sw * (common + kfac * ang_deriv<R>(rc, rb, ra, s1)) * irc;
                            if (smooth_on) {
                                sij -= dE0 * A.s.z * Bs.s.y * swjk;
                                sik -= dE0 * Bs.s.z * A.s.y * swjk;
                                sjk -= dE0 * dswjkr * A.s.y * Bs.s.y;
                            }
                            const R tij = triple * sij, tik = triple * sik, tjk = triple * sjk;
                            const R gx = tjk * vx, gy = tjk * vy, gz = tjk * vz;
                            // dE/dCN: root share here, partner shares through the entries
                            tde -= R(0.5) * dE * (A.c.y + Bs.c.y);
                            jacc[p][0] += tij;
                            jacc[p][1] -= gx; jacc[p][2] -= gy; jacc[p][3] -= gz;
                            jacc[p][4] -= R(0.5) * dE * (A.c.z + ejk.qrc);
                            kacc[q][0] += tik;
                            kacc[q][1] += gx; kacc[q][2] += gy; kacc[q][3] += gz;
                            kacc[q][4] -= R(0.5) * dE * (Bs.c.z + ejk.qcr);
                            txx += gx * vx; tyy += gy * vy; tzz += gz * vz;
                            txy += gx * vy; txz += gx * vz; tyz += gy * vz;
                        }
                    }
                    e_root += double(te);
                    if (GRAD) {
                        dei += double(tde);
                        sxx += double(txx); syy += double(tyy); szz += double(tzz);
                        sxy += double(txy); sxz += double(txz); syz += double(tyz);
                        // reduce the j-role sums over the 16 k-columns (half warp)
#pragma unroll
                        for (int p = 0; p < 2; p++)
#pragma unroll
                            for (int v = 0; v < kAcc; v++) {
                                R x = jacc[p][v];
                                x += __shfl_xor_sync(0xffffffffu, x, 8);
                                x += __shfl_xor_sync(0xffffffffu, x, 4);
                                x += __shfl_xor_sync(0xffffffffu, x, 2);
                                x += __shfl_xor_sync(0xffffffffu, x, 1);
                                jacc[p][v] = x;
                            }
                        if (tx == 0)
#pragma unroll
                            for (int p = 0; p < 2; p++) {
                                const int ka = A0 + ty + 16 * p;
                                if (ka < m)
                                    for (int v = 0; v < kAcc; v++) acc[ka * kAcc + v] += double(jacc[p][v]);
                            }
                    }
                }
                if (GRAD) {
                    // reduce the k-role sums over the 16 j-rows, half a k-tile at a time
#pragma unroll
                    for (int h = 0; h < 2; h++) {
                        __syncthreads();
#pragma unroll
                        for (int q = 0; q < 2; q++)
#pragma unroll
                            for (int v = 0; v < kAcc; v++) kred[ty][tx + 16 * q][v] = kacc[2 * h + q][v];
                        __syncthreads();
                        for (int k = tid; k < (kTB / 2) * kAcc; k += kThreadsAtm) {
                            const int ib = k / kAcc, v = k % kAcc;
                            const int slot = B0 + (kTB / 2) * h + ib;
                            if (slot >= m) continue;
                            double sum = 0.0;
                            for (int r = 0; r < 16; r++) sum += double(kred[r][ib][v]);
                            acc[slot * kAcc + v] += sum;
                        }
                    }
                }
            }
            __syncthreads();
        }
        // per-entry scatter: root share in registers, partner shares by FP64 atomics
        double gix = 0, giy = 0, giz = 0;
        if (GRAD && m > 0) {
            for (int k = tid; k < m; k += kThreadsAtm) {
                const double S = acc[k * kAcc + 0];
                const double Gx = acc[k * kAcc + 1], Gy = acc[k * kAcc + 2], Gz = acc[k * kAcc + 3];
                const double Dx = acc[k * kAcc + 4];
                if (S == 0.0 && Gx == 0.0 && Gy == 0.0 && Gz == 0.0 && Dx == 0.0) continue;
                const double4 v = nbr_v[base + k];
                const int x = nbr_j[base + k];
                gix -= S * v.x; giy -= S * v.y; giz -= S * v.z;
                atomicAdd(w.grad + 3 * x + 0, S * v.x + Gx);
                atomicAdd(w.grad + 3 * x + 1, S * v.y + Gy);
                atomicAdd(w.grad + 3 * x + 2, S * v.z + Gz);
                sxx += S * v.x * v.x; syy += S * v.y * v.y; szz += S * v.z * v.z;
                sxy += S * v.x * v.y; sxz += S * v.x * v.z; syz += S * v.y * v.z;
                atomicAdd(w.dEdcn + x, Dx);
            }
        }
        // block reduction of the root's sums in a fixed order
        double r[12] = {e_root, gix, giy, giz, dei, sxx, syy, szz, sxy, sxz, syz, double(ntrip)};
        for (int v = 0; v < 12; v++)
            for (int o = 16; o > 0; o >>= 1) r[v] += __shfl_xor_sync(0xffffffffu, r[v], o);
        if (lane == 0)
            for (int v = 0; v < 12; v++) wsum[tid >> 5][v] = r[v];
        __syncthreads();
        if (tid == 0) {
            double t[12] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
            for (int wq = 0; wq < kThreadsAtm / 32; wq++)
                for (int v = 0; v < 12; v++) t[v] += wsum[wq][v];
            e3[i] = t[0];
            if (w.counts) atomicAdd(w.counts + 1, (unsigned long long)t[11]);
            if (GRAD) {
                atomicAdd(w.grad + 3 * i + 0, t[1]);
                atomicAdd(w.grad + 3 * i + 1, t[2]);
                atomicAdd(w.grad + 3 * i + 2, t[3]);
                atomicAdd(w.dEdcn + i, t[4]);
                for (int v = 0; v < 6; v++) sig3[kSigma * i + v] = t[5 + v];
            }
        }
    }
}

}  // namespace

size_t atm_c6_entry_bytes(bool mixed) { return mixed ? sizeof(C6Entry<float>) : sizeof(C6Entry<double>); }

void launch_c6_matrix(const Batch& b, const Species& s, const Work& w, double alp3, const long long* d_mat_off,
                      void* mat, long long total, bool mixed, cudaStream_t stream)
{
    if (total <= 0) return;
    const int threads = 256;
    const long long blocks = (total + threads - 1) / threads;
    if (mixed) k_c6_matrix<float><<<(unsigned)blocks, threads, 0, stream>>>(b, s, w, alp3, d_mat_off, (C6Entry<float>*)mat, total);
    else k_c6_matrix<double><<<(unsigned)blocks, threads, 0, stream>>>(b, s, w, alp3, d_mat_off, (C6Entry<double>*)mat, total);
}

void launch_nbr_count(const Batch& b, const Config& c, const uint8_t* sys_skip, int* cnt, int* max_cnt,
                      cudaStream_t stream)
{
    if (b.natoms <= 0) return;
    k_nbr_count<<<(b.natoms + 7) / 8, 256, 0, stream>>>(b, c, sys_skip, cnt, max_cnt);
}

size_t scan_temp_bytes(int n)
{
    size_t bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, bytes, (const int*)nullptr, (long long*)nullptr, n + 1);
    return bytes;
}

void launch_scan(void* temp, size_t temp_bytes, const int* cnt_ext, long long* off, int n, cudaStream_t stream)
{
    // cnt_ext has n + 1 entries (last is 0): off[n] is the total
    cub::DeviceScan::ExclusiveSum(temp, temp_bytes, cnt_ext, off, n + 1, stream);
}

void launch_atm_guard(const long long* total, const int* max_cnt, long long cap, int stride, int* guard,
                      cudaStream_t stream)
{
    k_atm_guard<<<1, 1, 0, stream>>>(total, max_cnt, cap, stride, guard);
}

void launch_nbr_fill(const Batch& b, const Config& c, const uint8_t* sys_skip, const long long* off, int* nbr_j,
                     int* nbr_gend, double4* nbr_v, const int* guard, cudaStream_t stream)
{
    if (b.natoms <= 0) return;
    k_nbr_fill<<<(b.natoms + 7) / 8, 256, 0, stream>>>(b, c, sys_skip, off, nbr_j, nbr_gend, nbr_v, guard);
}

template <class R>
size_t triple_smem()
{
    return sizeof(Slot<R>) * (kTA + kTB) + sizeof(C6Entry<R>) * kTA * kTB + sizeof(R) * 16 * (kTB / 2) * kAcc;
}

template <class R, bool GRAD, bool PER>
int triple_occupancy_of()
{
    static bool configured = false;
    if (!configured) {
        cudaFuncSetAttribute(k_triples<R, GRAD, PER>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)triple_smem<R>());
        configured = true;
    }
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_triples<R, GRAD, PER>, kThreadsAtm, triple_smem<R>());
    return n > 0 ? n : 1;
}

template <class R, bool GRAD>
int triple_occupancy()
{
    // both variants are configured; the occupancy is the smaller of the two
    return std::min(triple_occupancy_of<R, GRAD, false>(), triple_occupancy_of<R, GRAD, true>());
}

int atm_blocks_per_sm(bool mixed, bool grad)
{
    if (mixed) return grad ? triple_occupancy<float, true>() : triple_occupancy<float, false>();
    return grad ? triple_occupancy<double, true>() : triple_occupancy<double, false>();
}

size_t atm_slot_bytes(bool mixed) { return mixed ? sizeof(Slot<float>) : sizeof(Slot<double>); }

template <class R, bool GRAD, bool PER>
void launch_triples_t(const Batch& b, const Species& s, const Damp& d, const Config& c, const Partition& p,
                      const Work& w, const void* mat, const long long* mat_off, const long long* off, const int* cnt,
                      const int* nbr_j, const int* nbr_gend, const double4* nbr_v, unsigned int* queue,
                      double* slot_acc, void* slot_scr, int slot_stride, int blocks, double* e3, double* sig3,
                      cudaStream_t stream)
{
    triple_occupancy_of<R, GRAD, PER>();
    k_triples<R, GRAD, PER><<<blocks, kThreadsAtm, triple_smem<R>(), stream>>>(
        b, s, d, c, p, w, (const C6Entry<R>*)mat, mat_off, off, cnt, nbr_j, nbr_gend, nbr_v, queue, slot_acc,
        (Slot<R>*)slot_scr, slot_stride, e3, sig3);
}

void launch_triples(const Batch& b, const Species& s, const Damp& d, const Config& c, const Partition& p,
                    const Work& w, const void* mat, const long long* mat_off, const long long* off, const int* cnt,
                    const int* nbr_j, const int* nbr_gend, const double4* nbr_v, unsigned int* queue,
                    double* slot_acc, void* slot_scr, int slot_stride, int blocks, bool periodic, double* e3,
                    double* sig3, cudaStream_t stream)
{
    if (b.natoms <= 0) return;
#define D3_TRIPLES(R, G, P)                                                                                  \
    launch_triples_t<R, G, P>(b, s, d, c, p, w, mat, mat_off, off, cnt, nbr_j, nbr_gend, nbr_v, queue, slot_acc, \
                              slot_scr, slot_stride, blocks, e3, sig3, stream)
    if (c.mixed) {
        if (c.grad) { if (periodic) D3_TRIPLES(float, true, true); else D3_TRIPLES(float, true, false); }
        else { if (periodic) D3_TRIPLES(float, false, true); else D3_TRIPLES(float, false, false); }
    } else {
        if (c.grad) { if (periodic) D3_TRIPLES(double, true, true); else D3_TRIPLES(double, true, false); }
        else { if (periodic) D3_TRIPLES(double, false, true); else D3_TRIPLES(double, false, false); }
    }
#undef D3_TRIPLES
}

}  // namespace d3
