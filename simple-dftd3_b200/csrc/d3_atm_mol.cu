// Axilrod-Teller-Muto three-body term for molecules: one block per system.
//
// For a non-periodic system of at most kMolMax atoms every triple is
// (i > j > k) in the sorted atom order (get_atm_dispersion_derivs,
// atm.f90:625-825, with a single lattice point, so triple_scale is 1).  A
// block takes the largest remaining molecule from a queue, stages its atoms
// in shared memory and hands out work items (root i, chunk of 32 rows j < i)
// to its warps.  A warp's lanes own one row j each; the warp sweeps the
// partners k < j in blocks of 32, whose (i, k) pair records the lanes build
// and share through shared memory.  Per triple the row keeps its j-role sums
// in registers, the k-role sums of the partners are reduced over the warp in
// groups of four with a reduce-scatter, and the root's sums stay in registers.  Per-atom
// gradient and dE/dCN accumulate in shared memory (FP64) and are added to the
// global arrays once per molecule; energy and virial are reduced per block
// in a fixed order.  No block-wide barrier separates the work items.
#include <cfloat>
#include <cstdint>

#include "d3_atm_common.cuh"
#include "d3_device.cuh"

namespace d3 {

namespace {

constexpr int kMolMax = 256;      // atoms of a system handled by one block
constexpr int kMolWarps = 8;
constexpr int kMolThreads = 32 * kMolWarps;

template <class R> struct V4;
template <> struct V4<float> { using type = float4; };
template <> struct V4<double> { using type = double4; };

// Record of the pair (root i, partner p).
template <class R>
struct PairRec {
    typename V4<R>::type h;   // absolute position of p (head in the mixed form), r_ip^2
    typename V4<R>::type l;   // tail of the position (mixed form), 1 / r_ip^2
    typename V4<R>::type c;   // sqrt(C6_ip), dC6_ip/dCN_i / C6_ip, dC6_ip/dCN_p / C6_ip, alp3 log(r0_ip / r_ip)
    typename V4<R>::type s;   // 1 / r_ip, switch, dsw/dr / r, valid (1 or 0)
};

template <class R>
__device__ __forceinline__ void split_pos(double x, R& h, R& l)
{
    if constexpr (sizeof(R) == 8) { h = x; l = 0.0; }
    else { h = __double2float_rn(x); l = __double2float_rn(x - (double)h); }
}

// Pair record of (i, p) from shared positions and the C6 row of i.
template <class R>
__device__ __forceinline__ PairRec<R> make_rec(const double* px, const double* py, const double* pz, int ii, int pp,
                                               bool in, const C6Entry<R>* row_i, R alp3, double cut2,
                                               bool smooth_on, R cutoff, R width)
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
        r.c.w = e.lr0 - 0.5 * (double)alp3 * log(r2s);
        r.l.w = 1.0 / r2s;
        r.s.x = rsqrt(r2s);
    } else {
        const float r2f = (float)r2s;
        r.c.w = e.lr0 - 0.5f * alp3 * __log2f(r2f);
        r.l.w = 1.0f / r2f;
        r.s.x = rsqrtf(r2f);
    }
    if (smooth_on && ok) {
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

template <class R, bool GRAD>
__global__ void __launch_bounds__(kMolThreads, sizeof(R) == 4 ? 2 : 1)
k_triples_mol(Batch b, Species sp, Damp d, Config c, Partition part, Work w, const C6Entry<R>* mat,
              const long long* mat_off, const int* mol_order, int nmol, unsigned int* queue, double* e3,
              double* sig3)
{
    extern __shared__ __align__(16) unsigned char smem[];
    double* px = reinterpret_cast<double*>(smem);
    double* py = px + kMolMax;
    double* pz = py + kMolMax;
    double* acc = pz + kMolMax;                                   // [kMolMax][4] gradient, dE/dCN
    PairRec<R>* recs = reinterpret_cast<PairRec<R>*>(acc + 4 * kMolMax);   // [warps][32]
    int* spc = reinterpret_cast<int*>(recs + kMolWarps * 32);     // [kMolMax] species
    int* loc = spc + kMolMax;                                     // [kMolMax] input index
    __shared__ double wred[kMolWarps][8];
    __shared__ int s_mol, s_item;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const R s9 = R(d.s9);
    const R alp = R(d.alp + 2.0);        // ATM exponent alp + 2 (rational.f90:563)
    const R alp3 = alp / R(3);
    const double cut2d = c.cut3 * c.cut3;
    const R cut2 = R(cut2d);
    const bool smooth_on = c.width3 > 0.0 && c.width3 < c.cut3;
    const R cutoff = R(c.cut3), width = R(c.width3);
    PairRec<R>* wrec = recs + wid * 32;

    for (;;) {
        __syncthreads();
        if (tid == 0) {
            const unsigned q = atomicAdd(queue, 1u);
            s_mol = q < (unsigned)nmol ? mol_order[q] : -1;
            s_item = 0;
        }
        __syncthreads();
        const int sys = s_mol;
        if (sys < 0) break;
        const int a0 = b.atom_off[sys];
        const int n = b.atom_off[sys + 1] - a0;
        const C6Entry<R>* m0 = mat + mat_off[sys];
        for (int a = tid; a < n; a += kMolThreads) {
            px[a] = b.x[a0 + a]; py[a] = b.y[a0 + a]; pz[a] = b.z[a0 + a];
            spc[a] = b.sp[a0 + a];
            loc[a] = b.local[a0 + a];
            acc[4 * a + 0] = 0.0; acc[4 * a + 1] = 0.0; acc[4 * a + 2] = 0.0; acc[4 * a + 3] = 0.0;
        }
        __syncthreads();
        const int nitems = n > 1 ? items_upto(n - 1) : 0;
        // per-lane sums over the warp's items: energy, virial, accepted triples
        double e_l = 0.0, sxx = 0, syy = 0, szz = 0, sxy = 0, sxz = 0, syz = 0;
        int ntrip = 0;
        for (;;) {
            int t = 0;
            if (lane == 0) t = atomicAdd(&s_item, 1);
            t = __shfl_sync(0xffffffffu, t, 0);
            if (t >= nitems) break;
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
            // root position split (head, tail)
            R rhx, rlx, rhy, rly, rhz, rlz;
            split_pos<R>(px[i], rhx, rlx);
            split_pos<R>(py[i], rhy, rly);
            split_pos<R>(pz[i], rhz, rlz);
            // this lane's row j
            const int j = 32 * chunk + lane;
            const bool jin = j < i;
            const int jj = jin ? j : 0;
            const PairRec<R> A = make_rec<R>(px, py, pz, i, jj, jin, row_i, alp3, cut2d, smooth_on, cutoff, width);
            const bool jvalid = A.s.w != R(0);
            if (!__any_sync(0xffffffffu, jvalid)) continue;
            const int kend = min(i, 32 * chunk + 32) - 1;   // partners k < j <= kend
            const int lj = loc[jj];
            const int li = loc[i];
            // j-role and root sums
            R jS = R(0), jGx = R(0), jGy = R(0), jGz = R(0), jD = R(0);
            R gix = R(0), giy = R(0), giz = R(0), dei = R(0);
            for (int K0 = 0; K0 < kend; K0 += 32) {
                const int kk = K0 + lane;
                const bool kin = kk < kend;
                const int kc = kin ? kk : 0;
                {
                    const PairRec<R> Bown = make_rec<R>(px, py, pz, i, kc, kin, row_i, alp3, cut2d, smooth_on, cutoff, width);
                    __syncwarp();
                    wrec[lane] = Bown;
                }
                __syncwarp();
                R kS = R(0), kGx = R(0), kGy = R(0), kGz = R(0), kD = R(0);
                R te = R(0), txx = R(0), tyy = R(0), tzz = R(0), txy = R(0), txz = R(0), tyz = R(0);
                const int tn = min(32, kend - K0);
                // one candidate (row j, partner K0 + tt): root, row and virial sums
                // here, the partner's five sums returned in cv
                auto candidate = [&](int tt, R* cv) {
                    R& cS = cv[0]; R& cGx = cv[1]; R& cGy = cv[2]; R& cGz = cv[3]; R& cD = cv[4];
                    const int k = K0 + tt;
                    const PairRec<R>& B = wrec[tt];
                    bool valid = jvalid && k < j && B.s.w != R(0);
                    // j-k vector from the absolute positions (head and tail differences)
                    R vx, vy, vz;
                    if constexpr (sizeof(R) == 8) {
                        vx = B.h.x - A.h.x; vy = B.h.y - A.h.y; vz = B.h.z - A.h.z;
                    } else {
                        vx = (B.h.x - A.h.x) + (B.l.x - A.l.x);
                        vy = (B.h.y - A.h.y) + (B.l.y - A.l.y);
                        vz = (B.h.z - A.h.z) + (B.l.z - A.l.z);
                    }
                    const R rc = vx * vx + vy * vy + vz * vz;
                    valid = valid && !(rc > cut2 || rc < R(DBL_EPSILON));
                    if (!__any_sync(0xffffffffu, valid)) return;
                    // C6 of (k, j): row k, column j (consecutive over the lanes)
                    const C6Entry<R> ekj = m0[(size_t)k * n + jj];
                    // a ghost gives C6 = 0 and with it zero contributions
                    if (valid && part.nparts > 1) {
                        // owner of the triple: the pair of its two largest input indices
                        int o1 = li, o2 = lj, o3 = loc[k], tmp;
                        if (o2 > o1) { tmp = o1; o1 = o2; o2 = tmp; }
                        if (o3 > o2) { tmp = o2; o2 = o3; o3 = tmp; }
                        if (o2 > o1) { tmp = o1; o1 = o2; o2 = tmp; }
                        valid = owns_pair_atm(part, o1, o2);
                    }
                    if (valid) {
                        const R ra = A.h.w, rb = B.h.w;           // r_ij^2, r_ik^2
                        const R rsc = rsqrt_r<R>(rc);
                        const R irc = rsc * rsc;
                        const R ir1 = A.s.x * B.s.x * rsc;        // 1 / (r_ij r_ik r_jk)
                        const R ir2 = ir1 * ir1;
                        const R ir3 = ir2 * ir1;
                        const R ir5 = ir3 * ir2;
                        // (r0/r1)^alp3 with r0 = r0ij r0ik r0jk, r1 = r_ij r_ik r_jk (atm.f90:744-749)
                        const R tq = rexp<R>(A.c.w + B.c.w + ekj.lr0 - R(0.5) * alp3 * rlog<R>(rc));
                        const R fdmp = rcp_r<R>(R(1) + R(6) * tq);
                        const R s1 = ra + rb + rc;
                        const R ang = R(0.375) * (s1 - R(2) * rb) * (s1 - R(2) * rc) * (s1 - R(2) * ra) * ir5 + ir3;
                        const R c9 = -s9 * A.c.x * B.c.x * ekj.sc6;
                        R sw = R(1), swjk = R(1), dswjkr = R(0);
                        if (smooth_on) {
                            R dsw;
                            const R rjk = rc * rsc;
                            smooth<R>(rjk, cutoff, width, swjk, dsw);
                            dswjkr = dsw * rsc;
                            sw = A.s.y * B.s.y * swjk;
                        }
                        const R dE0 = ang * fdmp * c9;
                        const R dE = dE0 * sw;
                        te -= dE;
                        ntrip++;
                        if (GRAD) {
                            const R common = c9 * ang * (R(-2) * alp * tq * (fdmp * fdmp));
                            const R kfac = R(0.375) * c9 * fdmp * ir5;
                            R sij = sw * (common + kfac * ang_deriv<R>(ra, rc, rb, s1)) * A.l.w;
                            R sik = sw * (common + kfac * ang_deriv<R>(rb, rc, ra, s1)) * B.l.w;
                            R sjk = sw * (common + kfac * ang_deriv<R>(rc, rb, ra, s1)) * irc;
                            if (smooth_on) {
                                sij -= dE0 * A.s.z * B.s.y * swjk;
                                sik -= dE0 * B.s.z * A.s.y * swjk;
                                sjk -= dE0 * dswjkr * A.s.y * B.s.y;
                            }
                            const R gx = sjk * vx, gy = sjk * vy, gz = sjk * vz;
                            // dE/dCN: root, row and partner shares (model.f90 dc6dcn / c6 ratios)
                            dei -= R(0.5) * dE * (A.c.y + B.c.y);
                            jS += sij; jGx -= gx; jGy -= gy; jGz -= gz;
                            jD -= R(0.5) * dE * (A.c.z + ekj.qcr);
                            cS = sik; cGx = gx; cGy = gy; cGz = gz;
                            cD = -R(0.5) * dE * (B.c.z + ekj.qrc);
                            txx += gx * vx; tyy += gy * vy; tzz += gz * vz;
                            txy += gx * vy; txz += gx * vz; tyz += gy * vz;
                        }
                    }
                };
                // partners in groups of four; their sums are reduced over the
                // warp with a reduce-scatter (10 + 5 + 3 x 5 shuffles for the
                // group) and handed to the partner's own lane
                for (int tg = 0; tg < tn; tg += 4) {
                    R kv[4][5];
#pragma unroll
                    for (int g = 0; g < 4; g++) {
#pragma unroll
                        for (int v = 0; v < 5; v++) kv[g][v] = R(0);
                        if (tg + g < tn) candidate(tg + g, kv[g]);
                    }
                    if (GRAD) {
                        const bool up16 = (lane & 16) != 0, up8 = (lane & 8) != 0;
                        R r2[2][5];
#pragma unroll
                        for (int h = 0; h < 2; h++)
#pragma unroll
                            for (int v = 0; v < 5; v++) {
                                const R send = up16 ? kv[h][v] : kv[2 + h][v];
                                const R keep = up16 ? kv[2 + h][v] : kv[h][v];
                                r2[h][v] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
                            }
                        R r1[5];
#pragma unroll
                        for (int v = 0; v < 5; v++) {
                            const R send = up8 ? r2[0][v] : r2[1][v];
                            const R keep = up8 ? r2[1][v] : r2[0][v];
                            r1[v] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
                        }
#pragma unroll
                        for (int v = 0; v < 5; v++)
#pragma unroll
                            for (int o = 4; o > 0; o >>= 1) r1[v] += __shfl_xor_sync(0xffffffffu, r1[v], o);
                        // lanes 16 b4 + 8 b3 + x now hold partner tg + 2 b4 + b3
                        const int gl = lane - tg;
                        const bool mine = gl >= 0 && gl < 4 && lane < tn;
                        const int src = mine ? 16 * (gl >> 1) + 8 * (gl & 1) : 0;
                        R got[5];
#pragma unroll
                        for (int v = 0; v < 5; v++) got[v] = __shfl_sync(0xffffffffu, r1[v], src);
                        if (mine) { kS += got[0]; kGx += got[1]; kGy += got[2]; kGz += got[3]; kD += got[4]; }
                    }
                }
                e_l += double(te);
                if (GRAD) {
                    sxx += double(txx); syy += double(tyy); szz += double(tzz);
                    sxy += double(txy); sxz += double(txz); syz += double(tyz);
                    // k-role of partner K0 + lane: pair (i, k) force along x_k - x_i
                    if (kin && (kS != R(0) || kGx != R(0) || kGy != R(0) || kGz != R(0) || kD != R(0))) {
                        const PairRec<R>& Bown = wrec[lane];
                        R vx, vy, vz;
                        if constexpr (sizeof(R) == 8) {
                            vx = Bown.h.x - rhx; vy = Bown.h.y - rhy; vz = Bown.h.z - rhz;
                        } else {
                            vx = (Bown.h.x - rhx) + (Bown.l.x - rlx);
                            vy = (Bown.h.y - rhy) + (Bown.l.y - rly);
                            vz = (Bown.h.z - rhz) + (Bown.l.z - rlz);
                        }
                        const double fx = double(kS * vx), fy = double(kS * vy), fz = double(kS * vz);
                        atomicAdd(acc + 4 * kk + 0, fx + double(kGx));
                        atomicAdd(acc + 4 * kk + 1, fy + double(kGy));
                        atomicAdd(acc + 4 * kk + 2, fz + double(kGz));
                        atomicAdd(acc + 4 * kk + 3, double(kD));
                        gix -= R(fx); giy -= R(fy); giz -= R(fz);
                        sxx += fx * vx; syy += fy * vy; szz += fz * vz;
                        sxy += fx * vy; sxz += fx * vz; syz += fy * vz;
                    }
                }
            }
            if (GRAD) {
                // row j: pair (i, j) force along x_j - x_i, and its partner sums
                if (jvalid) {
                    R vx, vy, vz;
                    if constexpr (sizeof(R) == 8) {
                        vx = A.h.x - rhx; vy = A.h.y - rhy; vz = A.h.z - rhz;
                    } else {
                        vx = (A.h.x - rhx) + (A.l.x - rlx);
                        vy = (A.h.y - rhy) + (A.l.y - rly);
                        vz = (A.h.z - rhz) + (A.l.z - rlz);
                    }
                    const double fx = double(jS * vx), fy = double(jS * vy), fz = double(jS * vz);
                    atomicAdd(acc + 4 * j + 0, fx + double(jGx));
                    atomicAdd(acc + 4 * j + 1, fy + double(jGy));
                    atomicAdd(acc + 4 * j + 2, fz + double(jGz));
                    atomicAdd(acc + 4 * j + 3, double(jD));
                    gix -= R(fx); giy -= R(fy); giz -= R(fz);
                    sxx += fx * vx; syy += fy * vy; szz += fz * vz;
                    sxy += fx * vy; sxz += fx * vz; syz += fy * vz;
                }
                const double rgx = wsum64(double(gix)), rgy = wsum64(double(giy)), rgz = wsum64(double(giz));
                const double rde = wsum64(double(dei));
                if (lane == 0) {
                    atomicAdd(acc + 4 * i + 0, rgx);
                    atomicAdd(acc + 4 * i + 1, rgy);
                    atomicAdd(acc + 4 * i + 2, rgz);
                    atomicAdd(acc + 4 * i + 3, rde);
                }
            }
        }
        // molecule totals: energy and virial in a fixed order, gradient and dE/dCN per atom
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
                w.grad[3 * (a0 + a) + 0] += acc[4 * a + 0];
                w.grad[3 * (a0 + a) + 1] += acc[4 * a + 1];
                w.grad[3 * (a0 + a) + 2] += acc[4 * a + 2];
                w.dEdcn[a0 + a] += acc[4 * a + 3];
            }
        }
    }
}

template <class R>
size_t mol_smem()
{
    return sizeof(double) * 3 * kMolMax + sizeof(double) * 4 * kMolMax + sizeof(PairRec<R>) * kMolWarps * 32 +
           sizeof(int) * 2 * kMolMax;
}

template <class R, bool GRAD>
void mol_configure()
{
    static bool configured = false;
    if (!configured) {
        cudaFuncSetAttribute(k_triples_mol<R, GRAD>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mol_smem<R>());
        configured = true;
    }
}

}  // namespace

int atm_mol_max_atoms() { return kMolMax; }

int atm_mol_blocks_per_sm(bool mixed, bool grad)
{
    int n = 0;
    if (mixed) {
        if (grad) { mol_configure<float, true>(); cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_triples_mol<float, true>, kMolThreads, mol_smem<float>()); }
        else { mol_configure<float, false>(); cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_triples_mol<float, false>, kMolThreads, mol_smem<float>()); }
    } else {
        if (grad) { mol_configure<double, true>(); cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_triples_mol<double, true>, kMolThreads, mol_smem<double>()); }
        else { mol_configure<double, false>(); cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_triples_mol<double, false>, kMolThreads, mol_smem<double>()); }
    }
    return n > 0 ? n : 1;
}

void launch_triples_mol(const Batch& b, const Species& s, const Damp& d, const Config& c, const Partition& p,
                        const Work& w, const void* mat, const long long* mat_off, const int* mol_order, int nmol,
                        unsigned int* queue, int blocks, double* e3, double* sig3, cudaStream_t stream)
{
    if (nmol <= 0) return;
    if (c.mixed) {
        const auto* m = (const C6Entry<float>*)mat;
        if (c.grad) {
            mol_configure<float, true>();
            k_triples_mol<float, true><<<blocks, kMolThreads, mol_smem<float>(), stream>>>(b, s, d, c, p, w, m, mat_off, mol_order, nmol, queue, e3, sig3);
        } else {
            mol_configure<float, false>();
            k_triples_mol<float, false><<<blocks, kMolThreads, mol_smem<float>(), stream>>>(b, s, d, c, p, w, m, mat_off, mol_order, nmol, queue, e3, sig3);
        }
    } else {
        const auto* m = (const C6Entry<double>*)mat;
        if (c.grad) {
            mol_configure<double, true>();
            k_triples_mol<double, true><<<blocks, kMolThreads, mol_smem<double>(), stream>>>(b, s, d, c, p, w, m, mat_off, mol_order, nmol, queue, e3, sig3);
        } else {
            mol_configure<double, false>();
            k_triples_mol<double, false><<<blocks, kMolThreads, mol_smem<double>(), stream>>>(b, s, d, c, p, w, m, mat_off, mol_order, nmol, queue, e3, sig3);
        }
    }
}

}  // namespace d3
