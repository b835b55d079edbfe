// Axilrod-Teller-Muto three-body term for molecules: one block per system.
//
// For a non-periodic system of at most kMolMax atoms every triple is
// (i > j > k) in the sorted atom order (get_atm_dispersion_derivs,
// atm.f90:625-825, with a single lattice point, so triple_scale is 1).  A
// block takes the largest remaining molecule from a queue and stages its
// atoms in shared memory.  The work items (root i, chunk of 32 rows j < i)
// are dealt to the warps round-robin in a fixed order.  A lane owns one row j
// and keeps the row's sums in registers; the partners k < j come in blocks
// of 32 whose (i, k) pair records the lanes build together.  Inside a block
// the warp walks the 32 x 32 (row, partner) tile along its diagonals: at step
// t lane l pairs row l with partner (l + t) mod 32, and the partner's five
// sums travel with the partner, one lane down per step (five shuffles), so
// that every lane ends the block holding one partner's complete sums.  In the
// diagonal block (the partners are the rows' own chunk) steps 1..16 visit
// every unordered pair once, which is enough because the triple term and its
// derivatives are symmetric in j and k.  Candidates are evaluated without
// branches: a term outside the cutoff gets weight zero.
//
// Per-atom gradient and dE/dCN go to per-warp FP64 accumulators in shared
// memory, summed over the warps in warp order at the end of the molecule;
// energy and virial are per-lane FP64 sums reduced in a fixed order.  With
// the fixed item order the result is bit-reproducible.
#include <algorithm>
#include <cfloat>
#include <cstdint>

#include "d3_atm_common.cuh"
#include "d3_device.cuh"

namespace d3 {

namespace {

constexpr int kMolMax = 256;      // atoms of a system handled by one block
constexpr int kMolWarps = 8;
constexpr int kMolThreads = 32 * kMolWarps;
#ifndef MOL_MINB
#define MOL_MINB 2
#endif

template <class R> struct V4;
template <> struct V4<float> { using type = float4; };
template <> struct V4<double> { using type = double4; };

// Record of the pair (root i, partner p).  An invalid record (p not a
// partner, or r_ip outside the cutoff) has sqrt(C6) = 0, valid = 0 and finite
// values elsewhere, so that a term built from it is finite and zero.
template <class R>
struct PairRec {
    typename V4<R>::type h;   // absolute position of p (head in the mixed form), r_ip^2
    typename V4<R>::type l;   // tail of the position (mixed form), 1 / r_ip^2
    typename V4<R>::type c;   // sqrt(C6_ip), dC6_ip/dCN_i / C6_ip, dC6_ip/dCN_p / C6_ip, alp3 log(r0_ip / r_ip)
    typename V4<R>::type s;   // 1 / r_ip, switch, dsw/dr / r, valid (1 or 0)
};

// Partner records of one warp, one array per field (the rotated reads of the
// lanes hit consecutive 16- or 32-byte slots).
template <class R>
struct MolTile {
    typename V4<R>::type h[32], l[32], c[32], s[32];
};

template <class R>
__device__ __forceinline__ void split_pos(double x, R& h, R& l)
{
    if constexpr (sizeof(R) == 8) { h = x; l = 0.0; }
    else { h = __double2float_rn(x); l = __double2float_rn(x - (double)h); }
}

// Pair record of (i, p) from shared positions and the C6 row of i.
template <class R, bool SMOOTH>
__device__ __forceinline__ PairRec<R> make_rec(const double* px, const double* py, const double* pz, int ii, int pp,
                                               bool in, const C6Entry<R>* row_i, R alp3, double cut2, R cutoff,
                                               R width)
{
    PairRec<R> r;
    const double x = px[pp], y = py[pp], z = pz[pp];
    const double vx = x - px[ii], vy = y - py[ii], vz = z - pz[ii];
    const double r2 = vx * vx + vy * vy + vz * vz;
    const bool ok = in && !(r2 > cut2 || r2 < DBL_EPSILON);
    R hx, lx, hy, ly, hz, lz;
    split_pos<R>(x, hx, lx);
    split_pos<R>(y, hy, ly);
    split_pos<R>(z, hz, lz);
    const double r2s = ok ? r2 : 1.0;
    const C6Entry<R> e = row_i[pp];
    r.h.x = hx; r.h.y = hy; r.h.z = hz; r.h.w = R(r2s);
    r.l.x = lx; r.l.y = ly; r.l.z = lz;
    r.c.x = ok ? e.sc6 : R(0); r.c.y = ok ? e.qrc : R(0); r.c.z = ok ? e.qcr : R(0);
    r.s.y = R(1); r.s.z = R(0); r.s.w = ok ? R(1) : R(0);
    // alp3 log(r0_ip / r_ip) with the damping radius term of the C6 entry,
    // 1 / r^2 and 1 / r: FP64, or FP32 from the FP64 distance in the mixed form
    if constexpr (sizeof(R) == 8) {
        r.c.w = ok ? e.lr0 - 0.5 * (double)alp3 * log(r2s) : 0.0;
        r.l.w = 1.0 / r2s;
        r.s.x = rsqrt(r2s);
    } else {
        const float r2f = (float)r2s;
        r.c.w = ok ? e.lr0 - 0.5f * alp3 * __log2f(r2f) : 0.0f;
        r.l.w = 1.0f / r2f;
        r.s.x = rsqrtf(r2f);
    }
    if (SMOOTH && ok) {
        R sw, dsw;
        const R rr = R(sqrt(r2s));
        smooth<R>(rr, cutoff, width, sw, dsw);
        r.s.y = sw;
        r.s.z = dsw / rr;
    }
    return r;
}

__device__ __forceinline__ double wsum64(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// S(x) = sum_{i=1..x} ceil(i / 32): work items of the roots 1..x.
__device__ __forceinline__ int items_upto(int x)
{
    const int q = x >> 5, r = x & 31;
    return 32 * (q * (q + 1) / 2) + r * (q + 1);
}

// Vector from the root to a record's position (head and tail differences).
template <class R>
__device__ __forceinline__ void root_vec(const typename V4<R>::type& h, const typename V4<R>::type& l, R rhx, R rhy,
                                         R rhz, R rlx, R rly, R rlz, R& vx, R& vy, R& vz)
{
    if constexpr (sizeof(R) == 8) {
        vx = h.x - rhx; vy = h.y - rhy; vz = h.z - rhz;
    } else {
        vx = (h.x - rhx) + (l.x - rlx);
        vy = (h.y - rhy) + (l.y - rly);
        vz = (h.z - rhz) + (l.z - rlz);
    }
}

// One work item (root i, chunk of 32 rows) of a molecule, by one warp: the
// triples (i, j, k) of the chunk's rows j with every k < j, added to the
// warp's per-atom accumulators acc[n][4] and to the lane's energy, virial and
// triple count.
template <class R, bool GRAD, bool SMOOTH>
__device__ __forceinline__ void mol_item(int t, int n, int nitems, const C6Entry<R>* m0, const double* px,
                                         const double* py, const double* pz, const int* loc, double* acc,
                                         MolTile<R>& tl, const Partition& part, R s9, R alp, R alp3, double cut2d,
                                         R cut2, R cutoff, R width, int lane, double& e_l, double& sxx, double& syy,
                                         double& szz, double& sxy, double& sxz, double& syz, int& ntrip)
{
        // item t -> root i (descending), chunk (descending within the root)
        const int u = nitems - t;
        int lo = 1, hi = n - 1;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (items_upto(mid) >= u) hi = mid; else lo = mid + 1;
        }
        const int i = lo;
        const int nch = (i + 31) >> 5;
        const int chunk = nch - 1 - (t - (nitems - items_upto(i)));
        const C6Entry<R>* row_i = m0 + (size_t)i * n;
        R rhx, rlx, rhy, rly, rhz, rlz;
        split_pos<R>(px[i], rhx, rlx);
        split_pos<R>(py[i], rhy, rly);
        split_pos<R>(pz[i], rhz, rlz);
        // this lane's row j
        const int J0 = 32 * chunk;
        const int j = J0 + lane;
        const bool jin = j < i;
        const int jj = jin ? j : 0;
        const PairRec<R> A = make_rec<R, SMOOTH>(px, py, pz, i, jj, jin, row_i, alp3, cut2d, cutoff, width);
        const bool jvalid = A.s.w != R(0);
        if (!__any_sync(0xffffffffu, jvalid)) return;
        const C6Entry<R>* row_j = m0 + (size_t)jj * n;
        const int lj = loc[jj];
        const int li = loc[i];
        // row and root sums of this lane, FP64 across partner blocks
        double jS = 0, jGx = 0, jGy = 0, jGz = 0, jD = 0, dei = 0, gix = 0, giy = 0, giz = 0;
        for (int K0 = 0; K0 <= J0; K0 += 32) {
            const bool diag = K0 == J0;
            // partner records k = K0 + lane (the rows' own records in the diagonal block)
            {
                PairRec<R> Bown;
                if (diag) Bown = A;
                else Bown = make_rec<R, SMOOTH>(px, py, pz, i, K0 + lane, true, row_i, alp3, cut2d, cutoff, width);
                __syncwarp();
                tl.h[lane] = Bown.h; tl.l[lane] = Bown.l; tl.c[lane] = Bown.c; tl.s[lane] = Bown.s;
            }
            __syncwarp();
            const int t0 = diag ? 1 : 0, t1 = diag ? 16 : 31;
            R kS = R(0), kGx = R(0), kGy = R(0), kGz = R(0), kD = R(0);
            R rS = R(0), rGx = R(0), rGy = R(0), rGz = R(0), rD = R(0), rde = R(0);
            R te = R(0), txx = R(0), tyy = R(0), tzz = R(0), txy = R(0), txz = R(0), tyz = R(0);
            // C6 of (j, k), in the FP32 form one step ahead of its use (the loads
            // overlap the arithmetic; the FP64 form has no registers to spare)
            auto c6_of = [&](int st) {
                const int k = K0 + ((lane + st) & 31);
                return row_j[k < n ? k : 0];
            };
            C6Entry<R> e_next = c6_of(t0);
            constexpr bool kPrefetch = sizeof(R) == 4;
            for (int st = t0; st <= t1; st++) {
                const int m = (lane + st) & 31;
                const typename V4<R>::type Bh = tl.h[m], Bl = tl.l[m], Bc = tl.c[m], Bs = tl.s[m];
                const int k = K0 + m;
                const int kc = k < n ? k : 0;
                // C6 of (j, k): qrc = dC6/dCN_j / C6, qcr = dC6/dCN_k / C6
                const C6Entry<R> ejk = kPrefetch ? e_next : c6_of(st);
                if (kPrefetch && st < t1) e_next = c6_of(st + 1);
                R vx, vy, vz;
                if constexpr (sizeof(R) == 8) {
                    vx = Bh.x - A.h.x; vy = Bh.y - A.h.y; vz = Bh.z - A.h.z;
                } else {
                    vx = (Bh.x - A.h.x) + (Bl.x - A.l.x);
                    vy = (Bh.y - A.h.y) + (Bl.y - A.l.y);
                    vz = (Bh.z - A.h.z) + (Bl.z - A.l.z);
                }
                const R rc0 = vx * vx + vy * vy + vz * vz;   // r_jk^2
                bool valid = jvalid && Bs.w != R(0) && (!diag || st < 16 || lane < 16) &&
                             !(rc0 > cut2 || rc0 < R(DBL_EPSILON));
                if (part.nparts > 1) {
                    // owner of the triple: the pair of its two largest input indices
                    int o1 = li, o2 = lj, o3 = loc[kc], tmp;
                    if (o2 > o1) { tmp = o1; o1 = o2; o2 = tmp; }
                    if (o3 > o2) { tmp = o2; o2 = o3; o3 = tmp; }
                    if (o2 > o1) { tmp = o1; o1 = o2; o2 = tmp; }
                    valid = valid && owns_pair_atm(part, o1, o2);
                }
                ntrip += valid ? 1 : 0;
                const R rc = valid ? rc0 : R(1);
                const R ra = A.h.w, rb = Bh.w;               // r_ij^2, r_ik^2
                const R rsc = rsqrt_r<R>(rc);
                const R irc = rsc * rsc;
                const R ir1 = A.s.x * Bs.x * rsc;            // 1 / (r_ij r_ik r_jk)
                const R ir2 = ir1 * ir1;
                const R ir3 = ir2 * ir1;
                const R ir5 = ir3 * ir2;
                // (r0/r1)^alp3 with r0 = r0ij r0ik r0jk, r1 = r_ij r_ik r_jk (atm.f90:744-749)
                const R tq = rexp<R>(A.c.w + Bc.w + ejk.lr0 - R(0.5) * alp3 * rlog<R>(rc));
                const R fdmp = rcp_r<R>(R(1) + R(6) * tq);
                const R s1 = ra + rb + rc;
                const R ang = R(0.375) * (s1 - R(2) * rb) * (s1 - R(2) * rc) * (s1 - R(2) * ra) * ir5 + ir3;
                const R c9 = valid ? -s9 * A.c.x * Bc.x * ejk.sc6 : R(0);
                R sw = R(1), swjk = R(1), dswjkr = R(0);
                if (SMOOTH) {
                    R dsw;
                    const R rjk = rc * rsc;
                    smooth<R>(rjk, cutoff, width, swjk, dsw);
                    dswjkr = dsw * rsc;
                    sw = A.s.y * Bs.y * swjk;
                }
                const R c9f = c9 * fdmp;
                const R dE0 = ang * c9f;
                const R dE = SMOOTH ? dE0 * sw : dE0;
                te -= dE;
                if (GRAD) {
                    const R common = dE0 * (R(-2) * alp * tq * fdmp);
                    const R kfac = R(0.375) * c9f * ir5;
                    R sij = (common + kfac * ang_deriv<R>(ra, rc, rb, s1)) * A.l.w;
                    R sik = (common + kfac * ang_deriv<R>(rb, rc, ra, s1)) * Bl.w;
                    R sjk = (common + kfac * ang_deriv<R>(rc, rb, ra, s1)) * irc;
                    if (SMOOTH) {
                        sij = sij * sw - dE0 * A.s.z * Bs.y * swjk;
                        sik = sik * sw - dE0 * Bs.z * A.s.y * swjk;
                        sjk = sjk * sw - dE0 * dswjkr * A.s.y * Bs.y;
                    }
                    const R gx = sjk * vx, gy = sjk * vy, gz = sjk * vz;
                    // dE/dCN shares of the root, the row and the partner
                    const R hdE = R(0.5) * dE;
                    rde -= hdE * (A.c.y + Bc.y);
                    rS += sij; rGx -= gx; rGy -= gy; rGz -= gz;
                    rD -= hdE * (A.c.z + ejk.qrc);
                    kS += sik; kGx += gx; kGy += gy; kGz += gz;
                    kD -= hdE * (Bc.z + ejk.qcr);
                    txx += gx * vx; tyy += gy * vy; tzz += gz * vz;
                    txy += gx * vy; txz += gx * vz; tyz += gy * vz;
                    // the partner's sums move one lane down, with the partner
                    const int src = (lane + 1) & 31;
                    kS = __shfl_sync(0xffffffffu, kS, src);
                    kGx = __shfl_sync(0xffffffffu, kGx, src);
                    kGy = __shfl_sync(0xffffffffu, kGy, src);
                    kGz = __shfl_sync(0xffffffffu, kGz, src);
                    kD = __shfl_sync(0xffffffffu, kD, src);
                }
            }
            e_l += double(te);
            if (GRAD) {
                sxx += double(txx); syy += double(tyy); szz += double(tzz);
                sxy += double(txy); sxz += double(txz); syz += double(tyz);
                jS += double(rS); jGx += double(rGx); jGy += double(rGy); jGz += double(rGz);
                jD += double(rD); dei += double(rde);
                // the lane now holds the sums of partner (lane + t1 + 1) mod 32:
                // its pair (i, k) force along x_k - x_i, and its jk and dE/dCN shares
                const int mf = (lane + t1 + 1) & 31;
                const int kk = K0 + mf;
                if (tl.s[mf].w != R(0)) {
                    R vx, vy, vz;
                    root_vec<R>(tl.h[mf], tl.l[mf], rhx, rhy, rhz, rlx, rly, rlz, vx, vy, vz);
                    const double fx = double(kS) * double(vx), fy = double(kS) * double(vy),
                                 fz = double(kS) * double(vz);
                    double* ak = acc + 4 * kk;
                    ak[0] += fx + double(kGx);
                    ak[1] += fy + double(kGy);
                    ak[2] += fz + double(kGz);
                    ak[3] += double(kD);
                    gix -= fx; giy -= fy; giz -= fz;
                    sxx += fx * double(vx); syy += fy * double(vy); szz += fz * double(vz);
                    sxy += fx * double(vy); sxz += fx * double(vz); syz += fy * double(vz);
                }
            }
        }
        if (GRAD) {
            // row j: pair (i, j) force along x_j - x_i, and the row's other sums
            if (jvalid) {
                R vx, vy, vz;
                root_vec<R>(A.h, A.l, rhx, rhy, rhz, rlx, rly, rlz, vx, vy, vz);
                const double fx = jS * double(vx), fy = jS * double(vy), fz = jS * double(vz);
                double* aj = acc + 4 * j;
                aj[0] += fx + jGx;
                aj[1] += fy + jGy;
                aj[2] += fz + jGz;
                aj[3] += jD;
                gix -= fx; giy -= fy; giz -= fz;
                sxx += fx * double(vx); syy += fy * double(vy); szz += fz * double(vz);
                sxy += fx * double(vy); sxz += fx * double(vz); syz += fy * double(vz);
            }
            const double rgx = wsum64(gix), rgy = wsum64(giy), rgz = wsum64(giz), rde = wsum64(dei);
            if (lane == 0) {
                double* ai = acc + 4 * i;
                ai[0] += rgx; ai[1] += rgy; ai[2] += rgz; ai[3] += rde;
            }
            __syncwarp();
        }
}

template <class R, bool GRAD, bool SMOOTH>
__global__ void __launch_bounds__(kMolThreads, sizeof(R) == 4 ? 2 : MOL_MINB)
k_triples_mol(Batch b, Species sp, Damp d, Config c, Partition part, Work w, const C6Entry<R>* mat,
              const long long* mat_off, const int* mol_order, int nmol, unsigned int* queue, double* e3,
              double* sig3)
{
    extern __shared__ __align__(16) unsigned char smem[];
    MolTile<R>* tiles = reinterpret_cast<MolTile<R>*>(smem);                   // [warps]
    double* accw = reinterpret_cast<double*>(tiles + kMolWarps);               // [warps][kMolMax][4]
    double* px = accw + (size_t)kMolWarps * kMolMax * 4;
    double* py = px + kMolMax;
    double* pz = py + kMolMax;
    int* loc = reinterpret_cast<int*>(pz + kMolMax);                           // [kMolMax] input index
    __shared__ double wred[kMolWarps][8];
    __shared__ int s_mol;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const R s9 = R(d.s9);
    const R alp = R(d.alp + 2.0);        // ATM exponent alp + 2 (rational.f90:563)
    const R alp3 = alp / R(3);
    const double cut2d = c.cut3 * c.cut3;
    const R cut2 = R(cut2d);
    const R cutoff = R(c.cut3), width = R(c.width3);
    MolTile<R>& tl = tiles[wid];
    double* acc = accw + (size_t)wid * kMolMax * 4;

    for (;;) {
        __syncthreads();
        if (tid == 0) {
            const unsigned q = atomicAdd(queue, 1u);
            s_mol = q < (unsigned)nmol ? mol_order[q] : -1;
        }
        __syncthreads();
        const int sys = s_mol;
        if (sys < 0) break;
        const int a0 = b.atom_off[sys];
        const int n = b.atom_off[sys + 1] - a0;
        const C6Entry<R>* m0 = mat + mat_off[sys];
        for (int a = tid; a < n; a += kMolThreads) {
            px[a] = b.x[a0 + a]; py[a] = b.y[a0 + a]; pz[a] = b.z[a0 + a];
            loc[a] = b.local[a0 + a];
        }
        if (GRAD)
            for (int a = tid; a < kMolWarps * n * 4; a += kMolThreads) {
                const int q = a / (n * 4);
                accw[(size_t)q * kMolMax * 4 + (a - q * n * 4)] = 0.0;
            }
        __syncthreads();
        const int nitems = n > 1 ? items_upto(n - 1) : 0;
        // per-lane sums over the warp's items: energy, virial, accepted triples
        double e_l = 0.0, sxx = 0, syy = 0, szz = 0, sxy = 0, sxz = 0, syz = 0;
        int ntrip = 0;
        for (int t = wid; t < nitems; t += kMolWarps)
            mol_item<R, GRAD, SMOOTH>(t, n, nitems, m0, px, py, pz, loc, acc, tl, part, s9, alp, alp3, cut2d, cut2,
                                      cutoff, width, lane, e_l, sxx, syy, szz, sxy, sxz, syz, ntrip);
        // molecule totals: energy and virial in a fixed order, gradient and
        // dE/dCN per atom summed over the warps in warp order
        double r[8] = {e_l, sxx, syy, szz, sxy, sxz, syz, double(ntrip)};
        for (int v = 0; v < 8; v++) r[v] = wsum64(r[v]);
        if (lane == 0)
            for (int v = 0; v < 8; v++) wred[wid][v] = r[v];
        __syncthreads();
        if (tid == 0) {
            double tot[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            for (int q = 0; q < kMolWarps; q++)
                for (int v = 0; v < 8; v++) tot[v] += wred[q][v];
            e3[a0] = tot[0];
            if (GRAD)
                for (int v = 0; v < 6; v++) sig3[kSigma * a0 + v] = tot[1 + v];
            if (w.counts) atomicAdd(w.counts + 1, (unsigned long long)tot[7]);
        }
        for (int a = tid; a < n; a += kMolThreads) {
            if (a > 0) {
                e3[a0 + a] = 0.0;
                if (GRAD)
                    for (int v = 0; v < 6; v++) sig3[kSigma * (a0 + a) + v] = 0.0;
            }
            if (GRAD) {
                double g0 = 0, g1 = 0, g2 = 0, g3 = 0;
                for (int q = 0; q < kMolWarps; q++) {
                    const double* aq = accw + ((size_t)q * kMolMax + a) * 4;
                    g0 += aq[0]; g1 += aq[1]; g2 += aq[2]; g3 += aq[3];
                }
                w.grad[3 * (a0 + a) + 0] += g0;
                w.grad[3 * (a0 + a) + 1] += g1;
                w.grad[3 * (a0 + a) + 2] += g2;
                w.dEdcn[a0 + a] += g3;
            }
        }
    }
}

template <class R>
size_t mol_smem()
{
    return sizeof(MolTile<R>) * kMolWarps + sizeof(double) * kMolWarps * kMolMax * 4 + sizeof(double) * 3 * kMolMax +
           sizeof(int) * kMolMax;
}

template <class R, bool GRAD, bool SMOOTH>
void mol_configure()
{
    static bool configured = false;
    if (!configured) {
        cudaFuncSetAttribute(k_triples_mol<R, GRAD, SMOOTH>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)mol_smem<R>());
        configured = true;
    }
}

template <class R, bool GRAD, bool SMOOTH>
int mol_occupancy()
{
    mol_configure<R, GRAD, SMOOTH>();
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_triples_mol<R, GRAD, SMOOTH>, kMolThreads, mol_smem<R>());
    return n;
}

template <class R, bool GRAD, bool SMOOTH>
void mol_launch(const Batch& b, const Species& s, const Damp& d, const Config& c, const Partition& p, const Work& w,
                const void* mat, const long long* mat_off, const int* mol_order, int nmol, unsigned int* queue,
                int blocks, double* e3, double* sig3, cudaStream_t stream)
{
    mol_configure<R, GRAD, SMOOTH>();
    k_triples_mol<R, GRAD, SMOOTH><<<blocks, kMolThreads, mol_smem<R>(), stream>>>(
        b, s, d, c, p, w, (const C6Entry<R>*)mat, mat_off, mol_order, nmol, queue, e3, sig3);
}

}  // namespace

int atm_mol_max_atoms() { return kMolMax; }

int atm_mol_blocks_per_sm(bool mixed, bool grad)
{
    // the smallest occupancy of the variants (the smooth-cutoff ones included)
    int n;
    if (mixed) {
        n = grad ? std::min(mol_occupancy<float, true, false>(), mol_occupancy<float, true, true>())
                 : std::min(mol_occupancy<float, false, false>(), mol_occupancy<float, false, true>());
    } else {
        n = grad ? std::min(mol_occupancy<double, true, false>(), mol_occupancy<double, true, true>())
                 : std::min(mol_occupancy<double, false, false>(), mol_occupancy<double, false, true>());
    }
    return n > 0 ? n : 1;
}

void launch_triples_mol(const Batch& b, const Species& s, const Damp& d, const Config& c, const Partition& p,
                        const Work& w, const void* mat, const long long* mat_off, const int* mol_order, int nmol,
                        unsigned int* queue, int blocks, double* e3, double* sig3, cudaStream_t stream)
{
    if (nmol <= 0) return;
    const bool smooth_on = c.width3 > 0.0 && c.width3 < c.cut3;
#define D3_MOL(R, G, S) mol_launch<R, G, S>(b, s, d, c, p, w, mat, mat_off, mol_order, nmol, queue, blocks, e3, sig3, stream)
    if (c.mixed) {
        if (c.grad) { if (smooth_on) D3_MOL(float, true, true); else D3_MOL(float, true, false); }
        else { if (smooth_on) D3_MOL(float, false, true); else D3_MOL(float, false, false); }
    } else {
        if (c.grad) { if (smooth_on) D3_MOL(double, true, true); else D3_MOL(double, true, false); }
        else { if (smooth_on) D3_MOL(double, false, true); else D3_MOL(double, false, false); }
    }
#undef D3_MOL
}

}  // namespace d3
