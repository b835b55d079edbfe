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

#include <cfloat>
#include <cstdint>

#include "d3_device.cuh"

namespace d3 {

namespace {

constexpr int kTA = 32;          // j-entries per tile
constexpr int kTB = 64;          // k-entries per tile
constexpr int kThreadsAtm = 256; // 16 x 16
constexpr int kAcc = 6;          // per-entry accumulators: S, D, Gx, Gy, Gz, Q
constexpr double kRs9 = 4.0 / 3.0;

// ------------------------------------------------------------ C6 matrix ----

template <class R>
struct C6Entry { R sc6, qrc, qcr; };

// {sqrt(C6_rc), dC6_rc/dCN_r / C6_rc, dC6_rc/dCN_c / C6_rc} for every ordered
// pair (r, c) of each system (get_atomic_c6, model.f90:432-461); ghosts give 0.
template <class R>
__global__ void k_c6_matrix(Batch b, Species s, Work w, const long long* mat_off, C6Entry<R>* mat,
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
    C6Entry<R> out{R(0), R(0), R(0)};
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
        if (c6 != 0.0) out = C6Entry<R>{R(sqrt(c6)), R(dr / c6), R(dc / c6)};
    }
    mat[t] = out;
}

// --------------------------------------------------------- neighbour lists --

__device__ __forceinline__ bool in_shell(double r2, double cut2) { return !(r2 > cut2 || r2 < DBL_EPSILON); }

// Number of entries (j <= i, T) with eps <= |x_j + T - x_i|^2 <= cutoff^2.
__global__ void k_nbr_count(Batch b, Config c, int* cnt, int* max_cnt)
{
    const int lane = threadIdx.x & 31;
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (i >= b.natoms) return;
    const int sys = b.sys_of_atom[i];
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

// Entries of root i in (j, T) order.  vec = (x_j + T) - x_i as in atm.f90:718.
__global__ void k_nbr_fill(Batch b, Config c, const long long* off, int* nbr_j, int* nbr_gend,
                           double4* nbr_v)
{
    const int lane = threadIdx.x & 31;
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (i >= b.natoms) return;
    const int sys = b.sys_of_atom[i];
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

template <class R>
__device__ __forceinline__ R rsqrt_r(R x) { if constexpr (sizeof(R) == 8) return sqrt(x); else return sqrtf(x); }

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

// One neighbour entry staged in shared memory.
template <class R>
struct Slot {
    R vx, vy, vz, r2;        // head of x_j + T - x_i and r^2
    float lx, ly, lz;        // tail of the vector (mixed form)
    R lr2;                   // log r^2 (base of rlog)
    R sc6, qij, qji;         // sqrt(C6_ij), dC6_ij/dCN_i / C6, dC6_ij/dCN_j / C6
    R lr0;                   // log(rs9 * rvdw_ij)
    R sw, dswr;              // switch and dsw/dr / r
    int atom, gend, sp, orig;
};

__device__ __forceinline__ bool owns_pair_atm(const Partition& p, int i, int j)
{
    long long hi = i > j ? i : j, lo = i > j ? j : i;
    return (hi * (hi + 1) / 2 + lo) % p.nparts == p.part;
}

template <class R>
__device__ __forceinline__ void load_slot(Slot<R>& s, int root, int k, long long base, const Batch& b,
                                          const Species& sp, const Config& c, const int* nbr_j,
                                          const int* nbr_gend, const double4* nbr_v, const C6Entry<R>* mat,
                                          long long mrow, int nsys_n, int a0)
{
    const int j = nbr_j[base + k];
    const double4 v = nbr_v[base + k];
    s.atom = j;
    s.gend = nbr_gend[base + k];
    s.sp = b.sp[j];
    s.orig = b.local[j];
    if constexpr (sizeof(R) == 8) {
        s.vx = v.x; s.vy = v.y; s.vz = v.z;
        s.lx = s.ly = s.lz = 0.f;
    } else {
        s.vx = __double2float_rn(v.x); s.vy = __double2float_rn(v.y); s.vz = __double2float_rn(v.z);
        s.lx = __double2float_rn(v.x - (double)s.vx);
        s.ly = __double2float_rn(v.y - (double)s.vy);
        s.lz = __double2float_rn(v.z - (double)s.vz);
    }
    s.r2 = R(v.w);
    s.lr2 = rlog<R>(R(v.w));
    const C6Entry<R> e = mat[mrow + (j - a0)];
    s.sc6 = e.sc6; s.qij = e.qrc; s.qji = e.qcr;
    const double r0 = __ldg(sp.atm_r0 + b.sp[root] * b.nid + s.sp);
    s.lr0 = rlog<R>(R(r0));
    if (c.width3 > 0.0 && c.width3 < c.cut3) {
        R sw, dsw;
        const R r = rsqrt_r<R>(R(v.w));
        smooth<R>(r, R(c.cut3), R(c.width3), sw, dsw);
        s.sw = sw; s.dswr = dsw / r;
    } else {
        s.sw = R(1); s.dswr = R(0);
    }
    (void)nsys_n;
}

template <class R, bool GRAD>
__global__ void __launch_bounds__(kThreadsAtm) k_triples(Batch b, Species sp, Damp d, Config c, Partition part,
                                                         Work w, const C6Entry<R>* mat, const long long* mat_off,
                                                         const long long* off, const int* cnt, const int* nbr_j,
                                                         const int* nbr_gend, const double4* nbr_v,
                                                         unsigned int* queue, double* slot_acc, int slot_stride,
                                                         double* e3, double* sig3)
{
    __shared__ Slot<R> sa[kTA];
    __shared__ Slot<R> sb[kTB];
    __shared__ R kred[16][kTB / 2][kAcc];
    __shared__ int s_root;
    const int tid = threadIdx.x;
    const int tx = tid & 15, ty = tid >> 4;
    const int lane = tid & 31;
    double* acc = slot_acc + (size_t)blockIdx.x * slot_stride * kAcc;
    const R s9 = R(d.s9);
    const R alp = R(d.alp + 2.0);        // ATM exponent alp + 2 (rational.f90:563)
    const R alp3 = alp / R(3);
    const R cut2 = R(c.cut3 * c.cut3);
    const bool smooth_on = c.width3 > 0.0 && c.width3 < c.cut3;
    const R cutoff = R(c.cut3), width = R(c.width3);
    // log-base conversion: rlog/rexp use base e (FP64) or base 2 (FP32)
    const R half = R(0.5);

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
        const long long mrow_i = mat_off[sys] + (long long)(i - a0) * nsys_n;
        const int orig_i = b.local[i];
        double e_root = 0.0;
        double sxx = 0, syy = 0, szz = 0, sxy = 0, sxz = 0, syz = 0;
        if (m > 0) {
            if (GRAD)
                for (int k = tid; k < m * kAcc; k += kThreadsAtm) acc[k] = 0.0;
            for (int B0 = 0; B0 < m; B0 += kTB) {
                __syncthreads();
                for (int k = tid; k < kTB; k += kThreadsAtm)
                    if (B0 + k < m)
                        load_slot<R>(sb[k], i, B0 + k, base, b, sp, c, nbr_j, nbr_gend, nbr_v, mat, mrow_i, nsys_n, a0);
                __syncthreads();
                // first j-entry whose group reaches this k-tile
                int astart = B0;
                while (astart > 0 && nbr_j[base + astart - 1] == nbr_j[base + B0]) astart--;
                R kacc[4][kAcc];
#pragma unroll
                for (int q = 0; q < 4; q++)
#pragma unroll
                    for (int v = 0; v < kAcc; v++) kacc[q][v] = R(0);
                for (int A0 = (astart / kTA) * kTA; A0 < m; A0 += kTA) {
                    __syncthreads();
                    for (int k = tid; k < kTA; k += kThreadsAtm)
                        if (A0 + k < m)
                            load_slot<R>(sa[k], i, A0 + k, base, b, sp, c, nbr_j, nbr_gend, nbr_v, mat, mrow_i, nsys_n, a0);
                    __syncthreads();
                    R jacc[2][kAcc];
#pragma unroll
                    for (int p = 0; p < 2; p++)
#pragma unroll
                        for (int v = 0; v < kAcc; v++) jacc[p][v] = R(0);
#pragma unroll
                    for (int p = 0; p < 2; p++) {
                        const int ia = ty + 16 * p;
                        if (A0 + ia >= m) continue;
                        const Slot<R>& A = sa[ia];
#pragma unroll
                        for (int q = 0; q < 4; q++) {
                            const int ib = tx + 16 * q;
                            const int kb = B0 + ib;
                            if (kb >= m || kb >= A.gend) continue;
                            const Slot<R>& Bs = sb[ib];
                            // j-k vector: (x_k + T_k - x_i) - (x_j + T_j - x_i)
                            R vx, vy, vz;
                            if constexpr (sizeof(R) == 8) {
                                vx = Bs.vx - A.vx; vy = Bs.vy - A.vy; vz = Bs.vz - A.vz;
                            } else {
                                vx = (Bs.vx - A.vx) + (Bs.lx - A.lx);
                                vy = (Bs.vy - A.vy) + (Bs.ly - A.ly);
                                vz = (Bs.vz - A.vz) + (Bs.lz - A.lz);
                            }
                            const R r2jk = vx * vx + vy * vy + vz * vz;
                            if (r2jk > cut2 || r2jk < R(DBL_EPSILON)) continue;
                            // C6 of the j-k pair
                            const int ja = A.atom, kb_atom = Bs.atom;
                            const C6Entry<R> ejk = mat[mat_off[sys] + (long long)(ja - a0) * nsys_n + (kb_atom - a0)];
                            if (GRAD && (A.sc6 == R(0) || Bs.sc6 == R(0) || ejk.sc6 == R(0))) continue;
                            if (part.nparts > 1) {
                                // owner of the triple: the pair of its two largest original indices
                                int o1 = orig_i, o2 = A.orig, o3 = Bs.orig, t;
                                if (o2 > o1) { t = o1; o1 = o2; o2 = t; }
                                if (o3 > o2) { t = o2; o2 = o3; o3 = t; }
                                if (o2 > o1) { t = o1; o1 = o2; o2 = t; }
                                if (!owns_pair_atm(part, o1, o2)) continue;
                            }
                            const R c9 = -s9 * A.sc6 * Bs.sc6 * ejk.sc6;
                            const R lr0jk = rlog<R>(R(__ldg(sp.atm_r0 + A.sp * b.nid + Bs.sp)));
                            const R r2ij = A.r2, r2ik = Bs.r2;
                            const R lr2jk = rlog<R>(r2jk);
                            // (r0/r1)^alp3 with r0 = r0ij r0ik r0jk, r1 = sqrt(r2ij r2ik r2jk)
                            const R r0r1 = rexp<R>(alp3 * ((A.lr0 + Bs.lr0 + lr0jk) - half * (A.lr2 + Bs.lr2 + lr2jk)));
                            const R r2 = r2ij * r2ik * r2jk;
                            const R r1 = rsqrt_r<R>(r2);
                            const R r3 = r2 * r1;
                            const R ir5 = R(1) / (r3 * r2);
                            const R fdmp = R(1) / (R(1) + R(6) * r0r1);
                            const R ang = R(0.375) * (r2ij + r2jk - r2ik) * (r2ij - r2jk + r2ik)
                                        * (-r2ij + r2jk + r2ik) * ir5 + r2 * ir5;
                            const R rr = ang * fdmp;
                            const int jat = A.atom, kat = Bs.atom;
                            R triple;
                            if (i == jat) triple = (i == kat) ? R(1.0 / 6.0) : R(0.5);
                            else triple = (i != kat && jat != kat) ? R(1) : R(0.5);
                            R sw = R(1);
                            R swjk = R(1), dswjkr = R(0);
                            if (smooth_on) {
                                R dsw;
                                const R rjk = rsqrt_r<R>(r2jk);
                                smooth<R>(rjk, cutoff, width, swjk, dsw);
                                dswjkr = dsw / rjk;
                                sw = A.sw * Bs.sw * swjk;
                            }
                            const R dE0 = rr * c9;
                            const R dE = dE0 * triple * sw;
                            e_root -= double(dE);
                            if (!GRAD) continue;
                            const R dfdmp = R(-2) * alp * r0r1 * (fdmp * fdmp);
                            const R base_ = c9 * ang * dfdmp;
                            // d/d r_ij, d/d r_ik, d/d r_jk of the angular term (atm.f90:751-776)
                            const R dang_ij = R(-0.375) * (r2ij * r2ij * r2ij + r2ij * r2ij * (r2jk + r2ik)
                                + r2ij * (R(3) * r2jk * r2jk + R(2) * r2jk * r2ik + R(3) * r2ik * r2ik)
                                - R(5) * (r2jk - r2ik) * (r2jk - r2ik) * (r2jk + r2ik)) * ir5;
                            const R dang_ik = R(-0.375) * (r2ik * r2ik * r2ik + r2ik * r2ik * (r2jk + r2ij)
                                + r2ik * (R(3) * r2jk * r2jk + R(2) * r2jk * r2ij + R(3) * r2ij * r2ij)
                                - R(5) * (r2jk - r2ij) * (r2jk - r2ij) * (r2jk + r2ij)) * ir5;
                            const R dang_jk = R(-0.375) * (r2jk * r2jk * r2jk + r2jk * r2jk * (r2ik + r2ij)
                                + r2jk * (R(3) * r2ik * r2ik + R(2) * r2ik * r2ij + R(3) * r2ij * r2ij)
                                - R(5) * (r2ik - r2ij) * (r2ik - r2ij) * (r2ik + r2ij)) * ir5;
                            R sij = sw * (base_ - c9 * dang_ij * fdmp) / r2ij;
                            R sik = sw * (base_ - c9 * dang_ik * fdmp) / r2ik;
                            R sjk = sw * (base_ - c9 * dang_jk * fdmp) / r2jk;
                            if (smooth_on) {
                                sij -= dE0 * A.dswr * Bs.sw * swjk;
                                sik -= dE0 * Bs.dswr * A.sw * swjk;
                                sjk -= dE0 * dswjkr * A.sw * Bs.sw;
                            }
                            const R tij = triple * sij, tik = triple * sik, tjk = triple * sjk;
                            const R gx = tjk * vx, gy = tjk * vy, gz = tjk * vz;
                            // j-role entry
                            jacc[p][0] += tij;
                            jacc[p][1] += dE;
                            jacc[p][2] -= gx; jacc[p][3] -= gy; jacc[p][4] -= gz;
                            jacc[p][5] += dE * ejk.qrc;
                            // k-role entry
                            kacc[q][0] += tik;
                            kacc[q][1] += dE;
                            kacc[q][2] += gx; kacc[q][3] += gy; kacc[q][4] += gz;
                            kacc[q][5] += dE * ejk.qcr;
                            // jk part of the virial
                            sxx += double(gx * vx); syy += double(gy * vy); szz += double(gz * vz);
                            sxy += double(gx * vy); sxz += double(gx * vz); syz += double(gy * vz);
                        }
                    }
                    if (GRAD) {
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
                    // reduce the k-role sums over the 16 j-rows of the block,
                    // half a k-tile at a time
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
        // per-entry scatter (fixed order per entry; atomics into partner atoms)
        double gix = 0, giy = 0, giz = 0, dei = 0;
        if (GRAD && m > 0) {
            for (int k = tid; k < m; k += kThreadsAtm) {
                const double S = acc[k * kAcc + 0], D = acc[k * kAcc + 1];
                const double Gx = acc[k * kAcc + 2], Gy = acc[k * kAcc + 3], Gz = acc[k * kAcc + 4];
                const double Q = acc[k * kAcc + 5];
                if (S == 0.0 && D == 0.0 && Gx == 0.0 && Gy == 0.0 && Gz == 0.0 && Q == 0.0) continue;
                const double4 v = nbr_v[base + k];
                const int x = nbr_j[base + k];
                const C6Entry<R> e = mat[mrow_i + (x - a0)];
                gix -= S * v.x; giy -= S * v.y; giz -= S * v.z;
                atomicAdd(w.grad + 3 * x + 0, S * v.x + Gx);
                atomicAdd(w.grad + 3 * x + 1, S * v.y + Gy);
                atomicAdd(w.grad + 3 * x + 2, S * v.z + Gz);
                sxx += S * v.x * v.x; syy += S * v.y * v.y; szz += S * v.z * v.z;
                sxy += S * v.x * v.y; sxz += S * v.x * v.z; syz += S * v.y * v.z;
                dei -= 0.5 * D * double(e.qrc);
                atomicAdd(w.dEdcn + x, -0.5 * (D * double(e.qcr) + Q));
            }
        }
        // block reduction of the root's sums in a fixed order
        double r[11] = {e_root, gix, giy, giz, dei, sxx, syy, szz, sxy, sxz, syz};
        for (int v = 0; v < 11; v++)
            for (int o = 16; o > 0; o >>= 1) r[v] += __shfl_xor_sync(0xffffffffu, r[v], o);
        __shared__ double wsum[8][11];
        if (lane == 0)
            for (int v = 0; v < 11; v++) wsum[tid >> 5][v] = r[v];
        __syncthreads();
        if (tid == 0) {
            double t[11] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
            for (int wq = 0; wq < kThreadsAtm / 32; wq++)
                for (int v = 0; v < 11; v++) t[v] += wsum[wq][v];
            e3[i] = t[0];
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

void launch_c6_matrix(const Batch& b, const Species& s, const Work& w, const long long* d_mat_off,
                      void* mat, long long total, bool mixed, cudaStream_t stream)
{
    if (total <= 0) return;
    const int threads = 256;
    const long long blocks = (total + threads - 1) / threads;
    if (mixed) k_c6_matrix<float><<<(unsigned)blocks, threads, 0, stream>>>(b, s, w, d_mat_off, (C6Entry<float>*)mat, total);
    else k_c6_matrix<double><<<(unsigned)blocks, threads, 0, stream>>>(b, s, w, d_mat_off, (C6Entry<double>*)mat, total);
}

void launch_nbr_count(const Batch& b, const Config& c, int* cnt, int* max_cnt, cudaStream_t stream)
{
    if (b.natoms <= 0) return;
    k_nbr_count<<<(b.natoms + 7) / 8, 256, 0, stream>>>(b, c, cnt, max_cnt);
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

void launch_nbr_fill(const Batch& b, const Config& c, const long long* off, int* nbr_j, int* nbr_gend,
                     double4* nbr_v, cudaStream_t stream)
{
    if (b.natoms <= 0) return;
    k_nbr_fill<<<(b.natoms + 7) / 8, 256, 0, stream>>>(b, c, off, nbr_j, nbr_gend, nbr_v);
}

int atm_blocks_per_sm(bool mixed, bool grad)
{
    int n = 0;
    if (mixed) {
        if (grad) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_triples<float, true>, kThreadsAtm, 0);
        else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_triples<float, false>, kThreadsAtm, 0);
    } else {
        if (grad) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_triples<double, true>, kThreadsAtm, 0);
        else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_triples<double, false>, kThreadsAtm, 0);
    }
    return n > 0 ? n : 1;
}

void launch_triples(const Batch& b, const Species& s, const Damp& d, const Config& c, const Partition& p,
                    const Work& w, const void* mat, const long long* mat_off, const long long* off, const int* cnt,
                    const int* nbr_j, const int* nbr_gend, const double4* nbr_v, unsigned int* queue,
                    double* slot_acc, int slot_stride, int blocks, double* e3, double* sig3, cudaStream_t stream)
{
    if (b.natoms <= 0) return;
    if (c.mixed) {
        if (c.grad)
            k_triples<float, true><<<blocks, kThreadsAtm, 0, stream>>>(b, s, d, c, p, w, (const C6Entry<float>*)mat, mat_off,
                off, cnt, nbr_j, nbr_gend, nbr_v, queue, slot_acc, slot_stride, e3, sig3);
        else
            k_triples<float, false><<<blocks, kThreadsAtm, 0, stream>>>(b, s, d, c, p, w, (const C6Entry<float>*)mat, mat_off,
                off, cnt, nbr_j, nbr_gend, nbr_v, queue, slot_acc, slot_stride, e3, sig3);
    } else {
        if (c.grad)
            k_triples<double, true><<<blocks, kThreadsAtm, 0, stream>>>(b, s, d, c, p, w, (const C6Entry<double>*)mat, mat_off,
                off, cnt, nbr_j, nbr_gend, nbr_v, queue, slot_acc, slot_stride, e3, sig3);
        else
            k_triples<double, false><<<blocks, kThreadsAtm, 0, stream>>>(b, s, d, c, p, w, (const C6Entry<double>*)mat, mat_off,
                off, cnt, nbr_j, nbr_gend, nbr_v, queue, slot_acc, slot_stride, e3, sig3);
    }
}


}  // namespace d3
