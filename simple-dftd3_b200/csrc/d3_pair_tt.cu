// Two-body dispersion over tile pairs, each unordered atom pair once.
//
// The sorted atoms of every system form tiles of 32 (d3_pair.cu).  A work
// unit is a pair of tiles (it >= jt) of one system; one warp evaluates it with
// one lane per atom i of tile it, while the partner atom j of tile jt and the
// lattice translation T are the same for the whole warp at each step.  The
// translations that can join the two tiles' bounding spheres within the
// cutoff are compacted per chunk of 128 into shared memory.  Every pair
// (i, j, T) of the reference's loop (rational.f90:438-514, zero.f90:455-553,
// mzero.f90:434-492, optimizedpower.f90:414-468, cso.f90:414-463,
// z.f90:405-450) is evaluated once: i's energy, virial and parameter-derivative shares hold
// both halves of the pair, i's gradient and dE/dCN stay in the lane, and j's
// gradient and dE/dCN are summed over the warp once per (chunk, j).  C6 and
// its CN derivatives come from per-atom species vectors
// U_j[s][r] = sum_r' C6ref(r, r', s, s_j) gw_j[r'] (get_atomic_c6,
// model.f90:432-461): seven multiply-adds per (i, j).  Each unit writes its
// per-lane sums to its own slots; a gather kernel adds the slots of every
// atom in a fixed order, so results are deterministic and no atomics are used.
#include <cfloat>
#include <cstdint>

#include "d3_device.cuh"
#include "d3_weights.cuh"

namespace d3 {

namespace {

constexpr int kTTWarps = 4;
constexpr int kTTThreads = 32 * kTTWarps;
constexpr int kTTChunk = 128;     // translations tested per pass
constexpr int kUnitI = 15;        // per-lane i sums: E, dE/dCN, g(3), sigma(6), dE/dparam(4)
constexpr int kUnitJ = 4;         // per-lane j sums: dE/dCN, g(3)
constexpr int kCnStore = 3;       // stored chain-rule sums per (i, j): countd (3)
constexpr double kKcnTT = 16.0;   // ncoord.f90:31
constexpr int kCnSigJ = 8;        // stored-sum CN pass: unit_i slots 8 .. 14 hold the j sums
                                  // (cn, countd v^T (6)) of the column atoms
constexpr int kSplitMax = 4;      // a unit is evaluated as 1, 2 (j-tile halves) or 4 items
                                  // (and translation halves); slots are sized for the largest split

template <class R> struct T4;
template <> struct T4<float> { using type = float4; };
template <> struct T4<double> { using type = double4; };

template <class R> __device__ __forceinline__ R tt_rcp(R x) { if constexpr (sizeof(R) == 8) return R(1) / x; else return __fdividef(1.0f, x); }
template <class R> __device__ __forceinline__ R tt_sqrt(R x) { if constexpr (sizeof(R) == 8) return sqrt(x); else return sqrtf(x); }
template <class R> __device__ __forceinline__ R tt_pow(R x, R a) { if constexpr (sizeof(R) == 8) return pow(x, a); else return powf(x, a); }

template <class R>
__device__ __forceinline__ void tt_smooth(R r, R cutoff, R width, R& sw, R& dswdr)
{
    // cutoff.f90:73-99
    if (width <= R(0) || width >= cutoff) { sw = R(1); dswdr = R(0); return; }
    const R inner = cutoff - width;
    if (r <= inner) { sw = R(1); dswdr = R(0); }
    else if (r >= cutoff) { sw = R(0); dswdr = R(0); }
    else {
        const R x = (cutoff - r) / width;
        sw = x * x * x * (R(10) + x * (R(-15) + R(6) * x));
        dswdr = R(-30) * x * x * (R(1) - x) * (R(1) - x) / width;
    }
}

__device__ __forceinline__ bool tt_owns(const Partition& p, int i, int j)
{
    // partition.f90:127-147 on system-local input indices
    if (p.nparts <= 1) return true;
    long long hi = i > j ? i : j, lo = i > j ? j : i;
    return (hi * (hi + 1) / 2 + lo) % p.nparts == p.part;
}

template <class R>
__device__ __forceinline__ R wsum_tt(R v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Warp sums of four values by a transposing butterfly (6 shuffles in place
// of 20): lane l returns the sum of value l >> 3 (a, b, c, d) over the warp.
template <class R>
__device__ __forceinline__ R wsum4_tt(R a, R b, R c, R d, int lane)
{
    const bool hi16 = lane & 16, hi8 = lane & 8;
    R x0 = hi16 ? c : a, x1 = hi16 ? d : b;
    const R y0 = hi16 ? a : c, y1 = hi16 ? b : d;
    x0 += __shfl_xor_sync(0xffffffffu, y0, 16);
    x1 += __shfl_xor_sync(0xffffffffu, y1, 16);
    R z = hi8 ? x1 : x0;
    const R y = hi8 ? x0 : x1;
    z += __shfl_xor_sync(0xffffffffu, y, 8);
    z += __shfl_xor_sync(0xffffffffu, z, 4);
    z += __shfl_xor_sync(0xffffffffu, z, 2);
    z += __shfl_xor_sync(0xffffffffu, z, 1);
    return z;
}

// The FP32 sweeps take two translations per step (the second masked off
// when a mask word has an odd count), branch-free, for instruction-level
// parallelism.  The FP64 sweeps, at the register limit, take one, and only
// the lanes whose term is taken run the FP64 math (its library sqrt, exp and
// divisions cost more issue slots than the divergence; measured on B200).
template <class R> constexpr bool kPairStep = sizeof(R) == 4;

// Distance vector v = x_i - x_j - T of a staged translation q (head and
// tail in the mixed form) and whether its term is taken: r^2 in [eps, cut2v]
// and `on`.  A term not taken gets r^2 = 1, so that the branch-free term
// math stays finite, and weight 0.
template <class R>
struct TTGeo {
    R vx, vy, vz, r2;
    bool ok;
};

template <class R, class V>
__device__ __forceinline__ TTGeo<R> tt_geo(const V* sth, const V* stl, int q, R dhx, R dhy, R dhz, R dlx, R dly,
                                           R dlz, R cut2v, R eps, bool on)
{
    TTGeo<R> g;
    const V th = sth[q];
    if constexpr (sizeof(R) == 8) { g.vx = dhx - th.x; g.vy = dhy - th.y; g.vz = dhz - th.z; }
    else {
        const V tl = stl[q];
        g.vx = (dhx - th.x) + (dlx - tl.x);
        g.vy = (dhy - th.y) + (dly - tl.y);
        g.vz = (dhz - th.z) + (dlz - tl.z);
    }
    const R r2 = g.vx * g.vx + g.vy * g.vy + g.vz * g.vz;
    g.ok = on && r2 <= cut2v && r2 >= eps;
    g.r2 = g.ok ? r2 : R(1);
    return g;
}

// Items of a unit: split 2 halves the j tile, split 4 also halves the
// translations; item sub of a unit takes j half sub % splitJ and
// translation half sub / splitJ.
__host__ __device__ __forceinline__ int tt_split_j(int split) { return split >= 2 ? 2 : 1; }

// Species vectors U and dU of one (atom, species) entry, padded to 8.
template <class R>
__device__ __forceinline__ void tt_load_uv(const R* p, R u[kRefPad], R du[kRefPad])
{
    if constexpr (sizeof(R) == 4) {
        const float4* q = reinterpret_cast<const float4*>(p);
        const float4 a0 = __ldg(q), a1 = __ldg(q + 1), b0 = __ldg(q + 2), b1 = __ldg(q + 3);
        u[0] = a0.x; u[1] = a0.y; u[2] = a0.z; u[3] = a0.w; u[4] = a1.x; u[5] = a1.y; u[6] = a1.z; u[7] = a1.w;
        du[0] = b0.x; du[1] = b0.y; du[2] = b0.z; du[3] = b0.w; du[4] = b1.x; du[5] = b1.y; du[6] = b1.z; du[7] = b1.w;
    } else {
        const double2* q = reinterpret_cast<const double2*>(p);
#pragma unroll
        for (int k = 0; k < kRefPad / 2; k++) {
            const double2 a = __ldg(q + k), b = __ldg(q + kRefPad / 2 + k);
            u[2 * k] = a.x; u[2 * k + 1] = a.y;
            du[2 * k] = b.x; du[2 * k + 1] = b.y;
        }
    }
}

// Compacts the translations tc .. tc+nt-1 that can join two tile spheres
// (centre difference dc, reach lim) into the warp's lists; returns their count.
template <class V>
__device__ __forceinline__ int tt_reach(const double* img, int tc, int nt, double dcx, double dcy, double dcz,
                                        double lim, int lane, V* sth, V* stl)
{
    int nreach = 0;
#pragma unroll
    for (int q = 0; q < kTTChunk / 32; q++) {
        const int k = 32 * q + lane;
        bool ok = false;
        double tx = 0, ty = 0, tz = 0;
        if (k < nt) {
            tx = __ldg(img + 3 * (tc + k)); ty = __ldg(img + 3 * (tc + k) + 1); tz = __ldg(img + 3 * (tc + k) + 2);
            const double ex = dcx - tx, ey = dcy - ty, ez = dcz - tz;
            ok = ex * ex + ey * ey + ez * ez <= lim * lim;
        }
        const unsigned m = __ballot_sync(0xffffffffu, ok);
        if (ok) {
            const int pos = nreach + __popc(m & ((1u << lane) - 1u));
            if constexpr (sizeof(V) == 32) {
                sth[pos] = make_double4(tx, ty, tz, 0.0);
            } else {
                const float hx = __double2float_rn(tx), hy = __double2float_rn(ty), hz = __double2float_rn(tz);
                sth[pos] = make_float4(hx, hy, hz, 0.f);
                stl[pos] = make_float4(__double2float_rn(tx - (double)hx), __double2float_rn(ty - (double)hy),
                                       __double2float_rn(tz - (double)hz), 0.f);
            }
        }
        nreach += __popc(m);
    }
    __syncwarp();
    return nreach;
}

constexpr int kJMaskWords = kTTChunk / 32;   // translations of an item, in ballot words

// Of the compacted translations [qbeg, qend), those that can bring atom j
// (position xj) within reach limj of the tile centre c: one bit each, in
// nwords = ceil((qend - qbeg) / 32) ballot words.  The test runs on the
// staged translations (head + tail, FP32 in the mixed form) with the reach
// widened by 1e-4 relative, so that it can only keep too many.
template <class V>
__device__ __forceinline__ int tt_jmask(const V* sth, const V* stl, int qbeg, int qend, double4 c, double xj,
                                        double yj, double zj, double limj, int lane, unsigned jm[kJMaskWords])
{
    const int nwords = (qend - qbeg + 31) / 32;
    using T = decltype(sth[0].x);
    const T ex0 = T(c.x - xj), ey0 = T(c.y - yj), ez0 = T(c.z - zj);
    const T lim2 = T(limj * limj * (1.0 + 2.0e-4));
#pragma unroll
    for (int h = 0; h < kJMaskWords; h++) {
        if (h >= nwords) { jm[h] = 0u; continue; }
        const int q = qbeg + 32 * h + lane;
        bool ok = false;
        if (q < qend) {
            const V th = sth[q];
            T ex = ex0 - th.x, ey = ey0 - th.y, ez = ez0 - th.z;
            if constexpr (sizeof(T) == 4) {
                const V tl = stl[q];
                ex -= tl.x; ey -= tl.y; ez -= tl.z;
            }
            ok = ex * ex + ey * ey + ez * ez <= lim2;
        }
        jm[h] = __ballot_sync(0xffffffffu, ok);
    }
    return nwords;
}

// Species vectors of every atom (sorted order): UV[a][s] = U[a][s][0..6], 0,
// dU[a][s][0..6], 0 (kRefPad stride, for vector loads).
template <class R>
__global__ void k_species_vectors(Batch b, Species s, Work w, R* UV)
{
    pdl_wait();
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long total = (long long)b.natoms * b.nid * kRefPad;
    if (t >= total) return;
    const int a = (int)(t / (b.nid * kRefPad));
    const int rem = (int)(t % (b.nid * kRefPad));
    const int sx = rem / kRefPad, r = rem % kRefPad;
    const int sa = b.sp[a];
    double u = 0.0, du = 0.0;
    if (!(b.ghost && b.ghost[a]) && r < s.nref[sx]) {
        const double* ref = s.c6ref + ((size_t)(sx * b.nid + sa) * kMaxRef + r) * kMaxRef;
        for (int q = 0; q < s.nref[sa]; q++) {
            u += w.gw[a * kMaxRef + q] * __ldg(ref + q);
            du += w.dgw[a * kMaxRef + q] * __ldg(ref + q);
        }
    }
    R* o = UV + ((size_t)a * b.nid + sx) * (2 * kRefPad);
    o[r] = R(u);
    o[kRefPad + r] = R(du);
}

// One (i, j, T) term of the modified zero, optimized power, CSO and Z forms:
// edisp0 and gdisp0 as the reference names them (E = -C6 edisp0 / 2 per
// half, gradient -C6 gdisp0 v) and, for Z damping, cdisp0 = d(C6 edisp0)/dC6.
// r1 is the distance when the smooth cutoff computed it.  Pair constants:
//   kMZero:          q1 = 1/(rs6 R0), q2 = 1/(rs8 R0), q3 = bet R0,
//                    q4 = rs6 bet R0^2, q5 = rs8 bet R0^2       (mzero.f90:441-472)
//   kOptimizedPower: q1 = R0^bet R0^6, q2 = R0^bet R0^8         (optimizedpower.f90:421-448)
//   kCSO:            q1 = (a3 sqrt(rrij) + a4)^6, q2 = a2 sqrt(rrij) (cso.f90:421-446)
//   kZDamping:       zc = a1 C6 / (species index sum)          (z.f90:412-431)
// The optimized power terms use r^-bet in place of the reference's
// r^bet / (r^bet r^6 + ...) and the CSO derivative 1 - sf = ef sf in the
// FP32 form, so that no intermediate leaves the FP32 range.
template <class R, int DAMP>
__device__ __forceinline__ void tt_family(R r2, R r1, bool have_r1, R rrij, R q1, R q2, R q3, R q4, R q5, R zc,
                                          R s6, R s8, R alp6, R alp8, R bet, R a1, R& edisp0, R& gdisp0,
                                          R& cdisp0)
{
    if constexpr (DAMP == kMZero) {
        if (!have_r1) r1 = tt_sqrt<R>(r2);
        const R r6 = r2 * r2 * r2;
        const R r8 = r6 * r2;
        const R t6 = tt_pow<R>(r1 * q1 + q3, -alp6);
        const R t8 = tt_pow<R>(r1 * q2 + q3, -alp8);
        const R f6 = R(1) / (R(1) + R(6) * t6);
        const R f8 = R(1) / (R(1) + R(6) * t8);
        const R d6 = R(-6) * f6 / r2 + R(6) * alp6 * t6 * (f6 * f6) / (r2 + q4 * r1);
        const R d8 = R(-8) * f8 / r2 + R(6) * alp8 * t8 * (f8 * f8) / (r2 + q5 * r1);
        edisp0 = s6 * f6 / r6 + s8 * rrij * f8 / r8;
        gdisp0 = s6 * d6 / r6 + s8 * rrij * d8 / r8;
    } else if constexpr (DAMP == kOptimizedPower) {
        // t6 = r^b / (r^b r^6 + q1) = 1 / (r^6 + q1 r^-b)
        const R ib = tt_pow<R>(r2, R(-0.5) * bet);
        const R r4 = r2 * r2;
        const R t6 = R(1) / (r4 * r2 + q1 * ib);
        const R t8 = R(1) / (r4 * r4 + q2 * ib);
        const R d6 = R(-6) * r4 * t6 * t6 + bet * q1 * t6 * t6 * ib / r2;
        const R d8 = R(-8) * r4 * r2 * t8 * t8 + bet * q2 * t8 * t8 * ib / r2;
        edisp0 = s6 * t6 + s8 * rrij * t8;
        gdisp0 = s6 * d6 + s8 * rrij * d8;
    } else if constexpr (DAMP == kCSO) {
        if (!have_r1) r1 = tt_sqrt<R>(r2);
        R sf, om;
        if constexpr (sizeof(R) == 8) {
            const R ef = exp(r1 - q2);
            sf = R(1) / (R(1) + ef);
            om = R(1) - sf;
        } else {
            const R ef = expf(fminf(r1 - q2, 80.f));
            sf = R(1) / (R(1) + ef);
            om = ef * sf;
        }
        const R sig = s6 + a1 * sf;
        const R r4 = r2 * r2;
        const R t6 = R(1) / (r4 * r2 + q1);
        const R dsig = -a1 * sf * om / r1;
        const R dt6 = R(-6) * r4 * t6 * t6;
        edisp0 = sig * t6;
        gdisp0 = dsig * t6 + sig * dt6;
    } else {
        const R r4 = r2 * r2;
        const R r6 = r4 * r2, r8 = r4 * r4;
        const R t6 = R(1) / (r6 + zc);
        const R t8 = R(1) / (r8 + zc * rrij);
        const R s8rr = s8 * rrij;
        edisp0 = s6 * t6 + s8rr * t8;
        gdisp0 = R(-6) * s6 * (r4 * t6) * t6 + R(-8) * s8rr * (r4 * r2 * t8) * t8;
        cdisp0 = s6 * (r6 * t6) * t6 + s8rr * (r8 * t8) * t8;
    }
}

// SMOOTH: the smooth cutoff of the two-body sum is on (0 < width < cutoff);
// a compile-time switch keeps its sqrt and divisions out of the plain loop.
// COUNT: the accepted terms are counted into w.counts (work counters only).
template <class R, int DAMP, bool GRAD, bool PG, bool SMOOTH, bool COUNT>
__global__ void __launch_bounds__(kTTThreads, sizeof(R) == 4 ? 4 : 3)
k_two_body_tt(Batch b, Species s, Damp d, Config c, Partition p, Work w, const int2* units, int nunits, int split,
              const R* UV, double* unit_i, double* unit_j)
{
    pdl_wait();
    using V = typename T4<R>::type;
    __shared__ V sth[kTTWarps][kTTChunk];
    __shared__ V stl[kTTWarps][kTTChunk];
    // FP64 sums, [value][lane]: i sums of the lane's atom, j sums of partner lane
    // (the FP64 form keeps its i sums in FP64 registers: j sums only)
    constexpr int kAccI = sizeof(R) == 4 ? kUnitI : 0;
    __shared__ double sacc[kTTWarps][kAccI + kUnitJ][32];
    // the reference weights gw, dgw/dCN of the lane's atom, [ref][lane]
    // (read once per partner)
    __shared__ R swt[kTTWarps][2 * kMaxRef][32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int item = blockIdx.x * kTTWarps + wid;
    if (item >= nunits * split) return;
    const int u = item / split, sub = item % split;
    const int splitJ = tt_split_j(split), splitT = split / splitJ;
    const int jh = sub % splitJ, th = sub / splitJ;
    const int it = units[u].x, jt = units[u].y;
    const int sys = b.tile_sys[it];
    const int t0 = b.tile_off[sys];
    const int as = b.atom_off[sys], ae = b.atom_off[sys + 1];
    const int ia0 = as + kTile * (it - t0), ja0 = as + kTile * (jt - t0);
    const int ni = min(kTile, ae - ia0), nj = min(kTile, ae - ja0);
    const bool diag = it == jt;
    const int i = ia0 + lane;
    const bool ivalid = lane < ni;
    const int ic = ivalid ? i : ia0;
    const int si = b.sp[ic], li = b.local[ic];
    const bool gi = b.ghost && b.ghost[ic];
    const double xi = b.x[ic], yi = b.y[ic], zi = b.z[ic];
    R hix, hiy, hiz, lix = R(0), liy = R(0), liz = R(0);
    if constexpr (sizeof(R) == 8) { hix = xi; hiy = yi; hiz = zi; }
    else {
        hix = __double2float_rn(xi); lix = __double2float_rn(xi - (double)hix);
        hiy = __double2float_rn(yi); liy = __double2float_rn(yi - (double)hiy);
        hiz = __double2float_rn(zi); liz = __double2float_rn(zi - (double)hiz);
    }
#pragma unroll
    for (int r = 0; r < kMaxRef; r++) {
        if constexpr (sizeof(R) == 8) {
            swt[wid][r][lane] = w.gw[ic * kMaxRef + r];
            swt[wid][kMaxRef + r][lane] = w.dgw[ic * kMaxRef + r];
        } else {
            swt[wid][r][lane] = w.gwf[ic * kMaxRef + r];
            swt[wid][kMaxRef + r][lane] = w.dgwf[ic * kMaxRef + r];
        }
    }
    const int tt0 = b.img_off[kImgDisp2 * (b.nsys + 1) + sys], tt1 = b.img_off[kImgDisp2 * (b.nsys + 1) + sys + 1];
    const double4 ci = b.tiles[it], cj = b.tiles[jt];
    const double lim = c.cut2 + ci.w + cj.w + 1.0e-6 * c.cut2 + 1.0e-6;
    const double limj = c.cut2 + ci.w + 1.0e-6 * c.cut2 + 1.0e-6;   // one atom j against tile it
    const double dcx = ci.x - cj.x, dcy = ci.y - cj.y, dcz = ci.z - cj.z;
    const R cutoff = R(c.cut2), cut2 = R(c.cut2 * c.cut2), width = R(c.width2);
    const R s6 = R(d.s6), s8 = R(d.s8);
    const R alp6 = R(d.alp), alp8 = R(d.alp + 2.0);
    const R bet = R(d.bet), a1 = R(d.a1);
    const int zsi = DAMP == kZDamping ? b.zid[ic] : 0;
    const int nid = b.nid;
    // i sums: FP32 form, partials in R over the partners of one translation
    // chunk (at most 32 additions), added to the FP64 sums in shared memory
    // per chunk; FP64 form, the register sums themselves
    double (*acc)[32] = sacc[wid];
    for (int v = 0; v < kAccI + kUnitJ; v++) acc[v][lane] = 0.0;
    __syncwarp();
    R te = R(0), tde = R(0), tgx = R(0), tgy = R(0), tgz = R(0);
    R txx = R(0), tyy = R(0), tzz = R(0), txy = R(0), txz = R(0), tyz = R(0);
    R tp0 = R(0), tp1 = R(0), tp2 = R(0), tp3 = R(0);
    unsigned nterm = 0;

    auto flush = [&]() {
        if constexpr (kAccI == 0) return;   // FP64 form: the register sums are the FP64 sums
        acc[0][lane] += double(te); acc[1][lane] += double(tde);
        te = tde = R(0);
        if (GRAD) {
            acc[2][lane] += double(tgx); acc[3][lane] += double(tgy); acc[4][lane] += double(tgz);
            acc[5][lane] += double(txx); acc[6][lane] += double(tyy); acc[7][lane] += double(tzz);
            acc[8][lane] += double(txy); acc[9][lane] += double(txz); acc[10][lane] += double(tyz);
            tgx = tgy = tgz = txx = tyy = tzz = txy = txz = tyz = R(0);
        }
        if (PG) {
            acc[11][lane] += double(tp0); acc[12][lane] += double(tp1);
            acc[13][lane] += double(tp2); acc[14][lane] += double(tp3);
            tp0 = tp1 = tp2 = tp3 = R(0);
        }
    };

    for (int tc = tt0; tc < tt1; tc += kTTChunk) {
        const int nt = min(kTTChunk, tt1 - tc);
        // translations that can join the two tiles
        const int nreach = tt_reach<V>(b.img, tc, nt, dcx, dcy, dcz, lim, lane, sth[wid], stl[wid]);
        if (nreach == 0) continue;
        // this item's part of the reachable translations
        const int qpart = (nreach + splitT - 1) / splitT;
        const int qbeg = th * qpart, qend = min(nreach, qbeg + qpart);
        if (qbeg >= qend) continue;
        const int jl0 = jh * (kTile / splitJ), jl1 = min(nj, jl0 + kTile / splitJ);
        for (int jl = jl0; jl < jl1; jl++) {
            const int j = ja0 + jl;
            const bool self = diag && jl == lane;
            bool valid = ivalid && (!diag || jl <= lane) && !gi;
            if (valid && p.nparts > 1) valid = tt_owns(p, li, b.local[j]);
            const int sj = b.sp[j];
            // C6 and its CN derivatives from the species vectors of j
            R c6 = R(0), dc6i = R(0), dc6j = R(0);
            if (valid) {
                R uj[kRefPad], duj[kRefPad];
                tt_load_uv<R>(UV + ((size_t)j * nid + si) * (2 * kRefPad), uj, duj);
#pragma unroll
                for (int r = 0; r < kMaxRef; r++) {
                    const R g = swt[wid][r][lane], dg = swt[wid][kMaxRef + r][lane];
                    c6 += g * uj[r];
                    dc6i += dg * uj[r];
                    dc6j += g * duj[r];
                }
                valid = c6 != R(0);
            }
            if (!__any_sync(0xffffffffu, valid)) continue;
            const double xj = b.x[j], yj = b.y[j], zj = b.z[j];
            R dhx, dhy, dhz, dlx = R(0), dly = R(0), dlz = R(0);
            if constexpr (sizeof(R) == 8) { dhx = xi - xj; dhy = yi - yj; dhz = zi - zj; }
            else {
                const float4 hj = b.xhi[j], lj4 = b.xlo[j];
                dhx = hix - hj.x; dhy = hiy - hj.y; dhz = hiz - hj.z;
                dlx = lix - lj4.x; dly = liy - lj4.y; dlz = liz - lj4.z;
            }
            const double2* pr = reinterpret_cast<const double2*>(s.pair + kPairSlots * (si * nid + sj));
            const double2 p01 = __ldg(pr), p23 = __ldg(pr + 1), p45 = __ldg(pr + 2);
            const R rrij = R(p01.x);
            const R q1 = R(p01.y), q2 = R(p23.x), q3 = R(p23.y), q4 = R(p45.x);
            const R q5 = DAMP == kMZero ? R(p45.y) : R(0);
            // Z damping: R0 C6 with R0 = a1 / (species index sum) (z.f90:413)
            const R zc = DAMP == kZDamping ? a1 / R(zsi + b.zid[j]) * c6 : R(0);
            // both halves of a pair go to i; a self pair (j = i, T != 0) is one half
            const R we = self ? R(0.5) : R(1);
            // a lane outside the pair list accepts no term
            const R cut2v = valid ? cut2 : R(-1);
            // sums over the translations of this (i, j); C6 and its derivatives,
            // which do not depend on T, multiply them afterwards
            R se = R(0), se6 = R(0), se8 = R(0), spa = R(0), spb = R(0);
            R sc = R(0);   // Z damping: sum of sw d(C6 edisp)/dC6, the factor of dC6/dCN
            R sgx = R(0), sgy = R(0), sgz = R(0);
            R sxx = R(0), syy = R(0), szz = R(0), sxy = R(0), sxz = R(0), syz = R(0);
            const R s8rr = s8 * rrij;
            // One (i, j, T) term, without branches: a lane whose term lies
            // outside the cutoff (or is the T = 0 self pair) evaluates it at
            // r^2 = 1 with weight 0 and adds exact zeros (tt_geo).
            auto geo = [&](int q, bool on) {
                return tt_geo<R, V>(sth[wid], stl[wid], q, dhx, dhy, dhz, dlx, dly, dlz, cut2v, R(DBL_EPSILON), on);
            };
            auto term = [&](const TTGeo<R>& g) {
                const R vx = g.vx, vy = g.vy, vz = g.vz, r2 = g.r2;
                const bool ok = g.ok;
                if constexpr (COUNT) nterm += ok ? 1u : 0u;
                // weight of the term; without the smooth cutoff the rational
                // form zeroes a rejected term through its reciprocal instead
                R sw = (SMOOTH || DAMP != kRational) ? (ok ? R(1) : R(0)) : R(1), dswdr = R(0), r1 = R(1);
                if constexpr (SMOOTH) {
                    r1 = tt_sqrt<R>(r2);
                    R sw1, dsw1;
                    tt_smooth<R>(r1, cutoff, width, sw1, dsw1);
                    sw = ok ? sw1 : R(0);
                    dswdr = ok ? dsw1 : R(0);
                }
                R edisp0, gdisp0, e6, e8, dpa = R(0), dpb = R(0), cdisp0 = R(0);
                if constexpr (DAMP == kRational) {
                    // rational.f90:462-497: q1 = R0^6, q2 = R0^8, q3 = R0, q4 = sqrt(rrij)
                    const R r4 = r2 * r2;
                    const R a6 = r4 * r2 + q1, a8 = r4 * r4 + q2;
                    const R inv = SMOOTH ? tt_rcp<R>(a6 * a8) : (ok ? tt_rcp<R>(a6 * a8) : R(0));
                    const R t6 = a8 * inv;
                    const R t8 = a6 * inv;
                    e6 = t6; e8 = rrij * t8;
                    edisp0 = s6 * t6 + s8rr * t8;
                    // s6 d6 + s8 rrij d8 with d6 = -6 r^4 t6^2, d8 = -8 r^6 t8^2
                    gdisp0 = r4 * (R(-6) * s6 * t6 * t6 + R(-8) * s8rr * r2 * t8 * t8);
                    if (PG) {
                        const R dedr0 = s6 * R(-6) * (q1 / q3) * t6 * t6 + s8rr * R(-8) * (q2 / q3) * t8 * t8;
                        dpa = dedr0 * q4;
                        dpb = dedr0;
                    }
                } else if constexpr (DAMP == kZero) {
                    // zero.f90:490-536: q1 = rs6 R0, q2 = rs8 R0
                    if (!SMOOTH) r1 = tt_sqrt<R>(r2);
                    const R r6 = r2 * r2 * r2;
                    const R r8 = r6 * r2;
                    const R t6 = tt_pow<R>(q1 / r1, alp6);
                    const R t8 = tt_pow<R>(q2 / r1, alp8);
                    const R f6 = R(1) / (R(1) + R(6) * t6);
                    const R f8 = R(1) / (R(1) + R(6) * t8);
                    const R d6 = R(-6) * f6 / r2 + R(6) * alp6 * t6 * (f6 * f6) / r2;
                    const R d8 = R(-8) * f8 / r2 + R(6) * alp8 * t8 * (f8 * f8) / r2;
                    e6 = f6 / r6; e8 = rrij * f8 / r8;
                    edisp0 = s6 * f6 / r6 + s8 * rrij * f8 / r8;
                    gdisp0 = s6 * d6 / r6 + s8 * rrij * d8 / r8;
                    if (PG) {
                        dpa = d.rs6 != 0.0 ? s6 / r6 * R(-6) * f6 * f6 * alp6 * t6 / R(d.rs6) : R(0);
                        dpb = d.rs8 != 0.0 ? s8 * rrij / r8 * R(-6) * f8 * f8 * alp8 * t8 / R(d.rs8) : R(0);
                    }
                } else {
                    e6 = e8 = R(0);
                    tt_family<R, DAMP>(r2, r1, SMOOTH, rrij, q1, q2, q3, q4, q5, zc, s6, s8, alp6, alp8, bet, a1,
                                       edisp0, gdisp0, cdisp0);
                }
                se += sw * edisp0;
                if (DAMP == kZDamping) sc += sw * cdisp0;
                if (PG) { se6 += sw * e6; se8 += sw * e8; spa += sw * dpa; spb += sw * dpb; }
                if (GRAD) {
                    R gdisp = sw * gdisp0;
                    if constexpr (SMOOTH) gdisp += dswdr * edisp0 / r1;
                    const R gx = gdisp * vx, gy = gdisp * vy, gz = gdisp * vz;
                    sgx += gx; sgy += gy; sgz += gz;
                    sxx += gx * vx; syy += gy * vy; szz += gz * vz;
                    sxy += gx * vy; sxz += gx * vz; syz += gy * vz;
                }
            };
            // translations of this part that can bring j within the cutoff of tile it
            unsigned jm[kJMaskWords];
            const int nw = tt_jmask<V>(sth[wid], stl[wid], qbeg, qend, ci, xj, yj, zj, limj, lane, jm);
#pragma unroll
            for (int h = 0; h < kJMaskWords; h++) {
                if (h >= nw) break;
                const int qh = qbeg + 32 * h - 1;
                for (unsigned mm = jm[h]; mm;) {
                    const int qa = qh + __ffs(mm);
                    mm &= mm - 1;
                    if constexpr (kPairStep<R>) {
                        const bool two = mm != 0u;
                        const int qb = two ? qh + __ffs(mm) : qa;
                        mm &= mm - 1;
                        const TTGeo<R> ga = geo(qa, true), gb = geo(qb, two);
                        term(ga);
                        term(gb);
                    } else {
                        const TTGeo<R> ga = geo(qa, true);
                        if (ga.ok) term(ga);
                    }
                }
            }
            // E_pair = -1/2 C6 edisp per half, dE/dCN = -dC6/dCN edisp, gradient -C6 gdisp v
            // (rational.f90:488-497); i takes both halves of E, sigma and dE/dparam
            const R c6w = c6 * we;
            te -= c6w * se;
            // dE/dCN = -dC6/dCN sum sw edisp; Z damping: dC6/dCN dE/dC6 (z.f90:431-445)
            const R sdc = DAMP == kZDamping ? sc : se;
            tde -= dc6i * sdc;
            const R jde = self ? R(0) : -dc6j * sdc;
            if (PG) { tp0 -= c6w * se6; tp1 -= c6w * se8; tp2 -= c6w * spa; tp3 -= c6w * spb; }
            if (GRAD) {
                R jgx = R(0), jgy = R(0), jgz = R(0);
                if (!self) {
                    tgx -= c6 * sgx; tgy -= c6 * sgy; tgz -= c6 * sgz;
                    jgx = c6 * sgx; jgy = c6 * sgy; jgz = c6 * sgz;
                }
                txx -= c6w * sxx; tyy -= c6w * syy; tzz -= c6w * szz;
                txy -= c6w * sxy; txz -= c6w * sxz; tyz -= c6w * syz;
                // j's share summed over the warp's atoms i: lane 8v holds value v
                const R z = wsum4_tt<R>(jde, jgx, jgy, jgz, lane);
                if ((lane & 7) == 0) acc[kAccI + (lane >> 3)][jl] += double(z);
            } else {
                const R z = wsum_tt<R>(jde);
                if (lane == 0) acc[kAccI][jl] += double(z);
            }
        }
        flush();
    }
    __syncwarp();
    double* oi = unit_i + ((size_t)item * kTile + lane) * kUnitI;
    if constexpr (kAccI > 0) {
        for (int v = 0; v < kUnitI; v++) oi[v] = acc[v][lane];
    } else {
        const double vi[kUnitI] = {double(te),  double(tde), double(tgx), double(tgy), double(tgz),
                                   double(txx), double(tyy), double(tzz), double(txy), double(txz),
                                   double(tyz), double(tp0), double(tp1), double(tp2), double(tp3)};
#pragma unroll
        for (int v = 0; v < kUnitI; v++) oi[v] = vi[v];
    }
    double* oj = unit_j + ((size_t)item * kTile + lane) * kUnitJ;
    for (int v = 0; v < kUnitJ; v++) oj[v] = acc[kAccI + v][lane];
    if (COUNT && w.counts) {
        unsigned long long n = nterm;
        for (int off = 16; off > 0; off >>= 1) n += __shfl_xor_sync(0xffffffffu, n, off);
        if (lane == 0) atomicAdd(w.counts + 0, n);
    }
}

// Two-body tile pairs of systems with the single lattice point T = 0
// (molecules), rational or zero damping with energy, dE/dCN, gradient and
// virial: one item per tile pair and no translation lists.  A warp walks the
// 32 x 32 (i, j) pairs along the diagonals: at step t lane l pairs atom
// ia0 + l with partner ja0 + (l + t) mod 32; the partner's dE/dCN and
// gradient sums move one lane down per step with the partner (four
// shuffles), so every lane ends the item holding one partner's sums.  The
// diagonal tile takes steps 1..16 (each unordered pair once; the i side takes
// the pair's energy and virial).  The slots are those of k_two_body_tt with
// one item per unit, so k_unit_gather adds them unchanged.  Compared with the
// general kernel, which runs each partner's translation list (one entry here),
// a step does one term without the per-partner reach mask and warp sums.
template <class R, int DAMP>
__global__ void __launch_bounds__(kTTThreads, sizeof(R) == 4 ? 4 : 3)
k_two_body_rot(Batch b, Species s, Damp d, Config c, Work w, const int2* units, int nunits, const R* UV,
               double* unit_i, double* unit_j)
{
    pdl_wait();
    using V = typename T4<R>::type;
    // per warp: the partner tile's positions (head, tail) and species
    __shared__ V sph[kTTWarps][kTile];
    __shared__ V spl[kTTWarps][kTile];
    __shared__ int ssp[kTTWarps][kTile];
    // pair constants per species pair: rrij, q1, q2, q3 (rational: R0^6, R0^8, R0;
    // zero: rs6 R0, rs8 R0, R0)
    __shared__ V spc[kMaxSpeciesFast * kMaxSpeciesFast];
    const int nid = b.nid;
    for (int k = threadIdx.x; k < nid * nid; k += kTTThreads) {
        const double* pr = s.pair + kPairSlots * k;
        if constexpr (sizeof(R) == 8) spc[k] = make_double4(pr[0], pr[1], pr[2], pr[3]);
        else spc[k] = make_float4(float(pr[0]), float(pr[1]), float(pr[2]), float(pr[3]));
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int item = blockIdx.x * kTTWarps + wid;
    if (item >= nunits) return;
    const int it = units[item].x, jt = units[item].y;
    const int sys = b.tile_sys[it];
    const int t0 = b.tile_off[sys];
    const int as = b.atom_off[sys], ae = b.atom_off[sys + 1];
    const int ia0 = as + kTile * (it - t0), ja0 = as + kTile * (jt - t0);
    const int ni = min(kTile, ae - ia0), nj = min(kTile, ae - ja0);
    const bool diag = it == jt;
    double* oi = unit_i + ((size_t)item * kTile + lane) * kUnitI;
    {
        // tile spheres farther apart than the cutoff: no pair, zero slots
        const double4 ci = b.tiles[it], cj = b.tiles[jt];
        const double dx = ci.x - cj.x, dy = ci.y - cj.y, dz = ci.z - cj.z;
        const double lim = c.cut2 + ci.w + cj.w + 1.0e-6 * c.cut2 + 1.0e-6;
        if (dx * dx + dy * dy + dz * dz > lim * lim) {
#pragma unroll
            for (int v = 0; v < kUnitI; v++) oi[v] = 0.0;
            double* oj = unit_j + ((size_t)item * kTile + lane) * kUnitJ;
#pragma unroll
            for (int v = 0; v < kUnitJ; v++) oj[v] = 0.0;
            return;
        }
    }
    const bool ivalid = lane < ni;
    const int ic = ivalid ? ia0 + lane : ia0;
    const int si = b.sp[ic];
    const bool gi = b.ghost && b.ghost[ic];
    const double xi = b.x[ic], yi = b.y[ic], zi = b.z[ic];
    R hix, hiy, hiz, lix = R(0), liy = R(0), liz = R(0);
    if constexpr (sizeof(R) == 8) { hix = xi; hiy = yi; hiz = zi; }
    else {
        hix = __double2float_rn(xi); lix = __double2float_rn(xi - (double)hix);
        hiy = __double2float_rn(yi); liy = __double2float_rn(yi - (double)hiy);
        hiz = __double2float_rn(zi); liz = __double2float_rn(zi - (double)hiz);
    }
    // the lane's reference weights
    R gwi[kMaxRef], dgwi[kMaxRef];
#pragma unroll
    for (int r = 0; r < kMaxRef; r++) {
        if constexpr (sizeof(R) == 8) { gwi[r] = w.gw[ic * kMaxRef + r]; dgwi[r] = w.dgw[ic * kMaxRef + r]; }
        else { gwi[r] = w.gwf[ic * kMaxRef + r]; dgwi[r] = w.dgwf[ic * kMaxRef + r]; }
    }
    // the partner tile: a partner outside the system (or a ghost) gets species -1
    {
        const bool jv = lane < nj;
        const int jc = jv ? ja0 + lane : ja0;
        if constexpr (sizeof(R) == 8) {
            sph[wid][lane] = make_double4(b.x[jc], b.y[jc], b.z[jc], 0.0);
        } else {
            sph[wid][lane] = b.xhi[jc];
            spl[wid][lane] = b.xlo[jc];
        }
        ssp[wid][lane] = (jv && !(b.ghost && b.ghost[jc])) ? b.sp[jc] : -1;
    }
    __syncwarp();
    const R cut2 = R(c.cut2 * c.cut2);
    const R s6 = R(d.s6), s8 = R(d.s8);
    const R alp6 = R(d.alp), alp8 = R(d.alp + 2.0);
    const bool iok = ivalid && !gi;
    const bool half = diag && lane >= 16;
    const int st0 = diag ? 1 : 0, st1 = diag ? 16 : 31;
    // i sums of the lane (FP32 partials in the mixed form), j sums travelling with the partner
    R te = R(0), tde = R(0), tgx = R(0), tgy = R(0), tgz = R(0);
    R txx = R(0), tyy = R(0), tzz = R(0), txy = R(0), txz = R(0), tyz = R(0);
    // the partner's sums travel in FP64 (a sum over the steps in order)
    double jde = 0.0, jgx = 0.0, jgy = 0.0, jgz = 0.0;
    for (int st = st0; st <= st1; st++) {
        const int m = (lane + st) & 31;
        const V ph = sph[wid][m];
        const int sj = ssp[wid][m];
        R vx, vy, vz;
        if constexpr (sizeof(R) == 8) { vx = hix - ph.x; vy = hiy - ph.y; vz = hiz - ph.z; }
        else {
            const V pl = spl[wid][m];
            vx = (hix - ph.x) + (lix - pl.x);
            vy = (hiy - ph.y) + (liy - pl.y);
            vz = (hiz - ph.z) + (liz - pl.z);
        }
        const R r2raw = vx * vx + vy * vy + vz * vz;
        const bool ok = iok && sj >= 0 && !(half && st == 16) && r2raw <= cut2 && r2raw >= R(DBL_EPSILON);
        // the FP32 form evaluates every lane (branch-free, a rejected term adds
        // zeros); the FP64 form only the lanes with a term (its library
        // division, sqrt and pow cost more than the divergence)
        if (sizeof(R) == 4 || ok) {
            const int sjc = sj >= 0 ? sj : 0;
            // C6 and its CN derivatives from the partner's species vectors for species si
            R u[kRefPad], du[kRefPad];
            tt_load_uv<R>(UV + ((size_t)(ja0 + (m < nj ? m : 0)) * nid + si) * (2 * kRefPad), u, du);
            R c6 = R(0), dc6i = R(0), dc6j = R(0);
#pragma unroll
            for (int r = 0; r < kMaxRef; r++) {
                c6 += gwi[r] * u[r];
                dc6i += dgwi[r] * u[r];
                dc6j += gwi[r] * du[r];
            }
            const V pc = spc[si * nid + sjc];
            const R rrij = pc.x, q1 = pc.y, q2 = pc.z;
            R edisp0, gdisp0;
            if constexpr (DAMP == kRational) {
                const R r2 = r2raw;
                const R r4 = r2 * r2;
                const R a6 = r4 * r2 + q1, a8 = r4 * r4 + q2;
                const R inv = ok ? tt_rcp<R>(a6 * a8) : R(0);
                const R t6 = a8 * inv;
                const R t8 = a6 * inv;
                const R s8rr = s8 * rrij;
                edisp0 = s6 * t6 + s8rr * t8;
                gdisp0 = r4 * (R(-6) * s6 * t6 * t6 + R(-8) * s8rr * r2 * t8 * t8);
            } else {
                // zero.f90:490-536 with q1 = rs6 R0, q2 = rs8 R0 (a rejected term at r^2 = 1, weight 0)
                const R r2 = ok ? r2raw : R(1);
                const R r1 = tt_sqrt<R>(r2);
                const R r6 = r2 * r2 * r2;
                const R r8 = r6 * r2;
                const R t6 = tt_pow<R>(q1 / r1, alp6);
                const R t8 = tt_pow<R>(q2 / r1, alp8);
                const R f6 = R(1) / (R(1) + R(6) * t6);
                const R f8 = R(1) / (R(1) + R(6) * t8);
                const R d6 = R(-6) * f6 / r2 + R(6) * alp6 * t6 * (f6 * f6) / r2;
                const R d8 = R(-8) * f8 / r2 + R(6) * alp8 * t8 * (f8 * f8) / r2;
                const R sw = ok ? R(1) : R(0);
                edisp0 = sw * (s6 * f6 / r6 + s8 * rrij * f8 / r8);
                gdisp0 = sw * (s6 * d6 / r6 + s8 * rrij * d8 / r8);
            }
            // E_pair = -C6 edisp (both halves to i), dE/dCN = -dC6/dCN edisp, gradient -C6 gdisp v
            // (rational.f90:488-497)
            te -= c6 * edisp0;
            tde -= dc6i * edisp0;
            jde -= double(dc6j * edisp0);
            const R f = c6 * gdisp0;
            const R gx = f * vx, gy = f * vy, gz = f * vz;
            tgx -= gx; tgy -= gy; tgz -= gz;
            jgx += double(gx); jgy += double(gy); jgz += double(gz);
            txx -= gx * vx; tyy -= gy * vy; tzz -= gz * vz;
            txy -= gx * vy; txz -= gx * vz; tyz -= gy * vz;
        }
        // the partner's sums move one lane down, with the partner
        const int src = (lane + 1) & 31;
        jde = __shfl_sync(0xffffffffu, jde, src);
        jgx = __shfl_sync(0xffffffffu, jgx, src);
        jgy = __shfl_sync(0xffffffffu, jgy, src);
        jgz = __shfl_sync(0xffffffffu, jgz, src);
    }
    const double vi[kUnitI] = {double(te),  double(tde), double(tgx), double(tgy), double(tgz),
                               double(txx), double(tyy), double(tzz), double(txy), double(txz),
                               double(tyz), 0.0,         0.0,         0.0,         0.0};
#pragma unroll
    for (int v = 0; v < kUnitI; v++) oi[v] = vi[v];
    // this lane holds the sums of partner (lane + st1 + 1) mod 32
    const int mf = (lane + st1 + 1) & 31;
    double* oj = unit_j + ((size_t)item * kTile + mf) * kUnitJ;
    oj[0] = jde; oj[1] = jgx; oj[2] = jgy; oj[3] = jgz;
}

// Coordination numbers of molecule tile pairs (the single lattice point
// T = 0; ncoord.f90:86-144) by the diagonal walk of k_two_body_rot, one item
// per tile pair.  STORE: also the chain rule's countd = dcf v / r of every
// (lane, step) into `store` (the slot of partner index st in the general
// kernel's layout) and the per-atom sums S of countd v^T on both sides; the
// partner's CN (and S) travel with the partner, in FP64 (a sum over the
// steps in order, not a tree, would lose more in FP32 than the terms do).
// Slots as k_cn_tt<R, 0 or 2>.
template <class R, bool STORE>
__global__ void __launch_bounds__(kTTThreads)
k_cn_rot(Batch b, Species s, Config c, Work w, const int2* units, int nunits, double* unit_i, double* unit_j,
         R* store, unsigned char* store_ok)
{
    pdl_wait();
    using V = typename T4<R>::type;
    __shared__ V sph[kTTWarps][kTile];
    __shared__ V spl[kTTWarps][kTile];
    __shared__ double srj[kTTWarps][kTile];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int item = blockIdx.x * kTTWarps + wid;
    if (item >= nunits) return;
    const int it = units[item].x, jt = units[item].y;
    const int sys = b.tile_sys[it];
    const int t0 = b.tile_off[sys];
    const int as = b.atom_off[sys], ae = b.atom_off[sys + 1];
    const int ia0 = as + kTile * (it - t0), ja0 = as + kTile * (jt - t0);
    const int ni = min(kTile, ae - ia0), nj = min(kTile, ae - ja0);
    const bool diag = it == jt;
    double* oi = unit_i + ((size_t)item * kTile + lane) * kUnitI;
    {
        // tile spheres farther apart than the cutoff: no term, zero slots
        const double4 ci = b.tiles[it], cj = b.tiles[jt];
        const double dx = ci.x - cj.x, dy = ci.y - cj.y, dz = ci.z - cj.z;
        const double lim = c.cut_cn + ci.w + cj.w + 1.0e-6 * c.cut_cn + 1.0e-6;
        if (dx * dx + dy * dy + dz * dz > lim * lim) {
            if (STORE) {
#pragma unroll
                for (int v = 0; v < 7; v++) { oi[v] = 0.0; oi[kCnSigJ + v] = 0.0; }
                if (lane == 0) store_ok[item] = 0;
            } else {
                oi[0] = 0.0;
                unit_j[((size_t)item * kTile + lane) * kUnitJ] = 0.0;
            }
            return;
        }
    }
    const bool ivalid = lane < ni;
    const int ic = ivalid ? ia0 + lane : ia0;
    const double rci = s.rcov[b.sp[ic]];
    const double xi = b.x[ic], yi = b.y[ic], zi = b.z[ic];
    R hix, hiy, hiz, lix = R(0), liy = R(0), liz = R(0);
    if constexpr (sizeof(R) == 8) { hix = xi; hiy = yi; hiz = zi; }
    else {
        hix = __double2float_rn(xi); lix = __double2float_rn(xi - (double)hix);
        hiy = __double2float_rn(yi); liy = __double2float_rn(yi - (double)hiy);
        hiz = __double2float_rn(zi); liz = __double2float_rn(zi - (double)hiz);
    }
    {
        // the partner tile: positions, covalent radius (a partner outside the system: -1)
        const bool jv = lane < nj;
        const int jc = jv ? ja0 + lane : ja0;
        srj[wid][lane] = jv ? s.rcov[b.sp[jc]] : -1.0;
        if constexpr (sizeof(R) == 8) {
            sph[wid][lane] = make_double4(b.x[jc], b.y[jc], b.z[jc], 0.0);
        } else {
            sph[wid][lane] = b.xhi[jc];
            spl[wid][lane] = b.xlo[jc];
        }
    }
    __syncwarp();
    const R cut2 = R(c.cut_cn * c.cut_cn);
    const bool half = diag && lane >= 16;
    const int st0 = diag ? 1 : 0, st1 = diag ? 16 : 31;
    double cn_i = 0.0;
    double sxx = 0, syy = 0, szz = 0, sxy = 0, sxz = 0, syz = 0;
    double cn_j = 0.0, jxx = 0, jyy = 0, jzz = 0, jxy = 0, jxz = 0, jyz = 0;
    for (int st = st0; st <= st1; st++) {
        const int m = (lane + st) & 31;
        const V ph = sph[wid][m];
        R vx, vy, vz;
        if constexpr (sizeof(R) == 8) { vx = hix - ph.x; vy = hiy - ph.y; vz = hiz - ph.z; }
        else {
            const V pl = spl[wid][m];
            vx = (hix - ph.x) + (lix - pl.x);
            vy = (hiy - ph.y) + (liy - pl.y);
            vz = (hiz - ph.z) + (liz - pl.z);
        }
        const R r2 = vx * vx + vy * vy + vz * vz;
        const double rcj = srj[wid][m];
        const bool ok = ivalid && rcj >= 0.0 && !(half && st == 16) && r2 <= cut2 && r2 >= R(1.0e-12);
        R cf = R(0), f = R(0);
        // the FP32 form evaluates every lane (a rejected term adds zeros); the
        // FP64 form only the lanes with a term
        if (sizeof(R) == 4 || ok) {
            const R rc = R(rci + rcj);
            const R rr = ok ? r2 : R(1);
            if constexpr (sizeof(R) == 8) {
                const R r1 = sqrt(rr);
                cf = R(1) / (R(1) + exp(-R(kKcnTT) * (rc / r1 - R(1))));
                f = -cf * (R(1) - cf) * R(kKcnTT) * rc / rr / r1;
            } else {
                const R ir = rsqrtf(rr);
                cf = __fdividef(1.0f, 1.0f + expf(-R(kKcnTT) * (rc * ir - R(1))));
                f = -cf * (R(1) - cf) * R(kKcnTT) * rc * (ir * ir * ir);
            }
            cf = ok ? cf : R(0);
            f = ok ? f : R(0);
        }
        cn_i += double(cf);
        cn_j += double(cf);
        if (STORE) {
            const R cx = f * vx, cy = f * vy, cz = f * vz;   // countd
            R* out = store + ((size_t)item * kTile + st) * kCnStore * kTile + lane;
            out[0] = cx; out[kTile] = cy; out[2 * kTile] = cz;
            const double qxx = double(cx * vx), qyy = double(cy * vy), qzz = double(cz * vz);
            const double qxy = double(cx * vy), qxz = double(cx * vz), qyz = double(cy * vz);
            sxx += qxx; syy += qyy; szz += qzz; sxy += qxy; sxz += qxz; syz += qyz;
            jxx += qxx; jyy += qyy; jzz += qzz; jxy += qxy; jxz += qxz; jyz += qyz;
        }
        // the partner's sums move one lane down, with the partner
        const int src = (lane + 1) & 31;
        cn_j = __shfl_sync(0xffffffffu, cn_j, src);
        if (STORE) {
            jxx = __shfl_sync(0xffffffffu, jxx, src); jyy = __shfl_sync(0xffffffffu, jyy, src);
            jzz = __shfl_sync(0xffffffffu, jzz, src); jxy = __shfl_sync(0xffffffffu, jxy, src);
            jxz = __shfl_sync(0xffffffffu, jxz, src); jyz = __shfl_sync(0xffffffffu, jyz, src);
        }
    }
    // this lane holds the sums of partner (lane + st1 + 1) mod 32
    const int mf = (lane + st1 + 1) & 31;
    if (STORE) {
        // (k_cn_chain_rot reads the steps the walk took only)
        oi[0] = cn_i;
        oi[1] = sxx; oi[2] = syy; oi[3] = szz; oi[4] = sxy; oi[5] = sxz; oi[6] = syz;
        double* oj = unit_i + ((size_t)item * kTile + mf) * kUnitI + kCnSigJ;
        oj[0] = cn_j;
        oj[1] = jxx; oj[2] = jyy; oj[3] = jzz;
        oj[4] = jxy; oj[5] = jxz; oj[6] = jyz;
        if (lane == 0) store_ok[item] = 1;
    } else {
        oi[0] = cn_i;
        unit_j[((size_t)item * kTile + mf) * kUnitJ] = cn_j;
    }
}

// CN chain rule gradient of molecule tile pairs from the sums k_cn_rot<R, true>
// stored, by the same walk: per (lane, step) the weight dE/dCN_i + dE/dCN_j
// times the stored countd (ncoord.f90:205-209); the partner's gradient sums
// travel with the partner.  Slots as k_cn_chain_stored.
template <class R>
__global__ void __launch_bounds__(kTTThreads)
k_cn_chain_rot(Batch b, Work w, const int2* units, int nunits, const R* store, const unsigned char* store_ok,
               double* unit_i, double* unit_j)
{
    pdl_wait();
    __shared__ double sde[kTTWarps][kTile];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int item = blockIdx.x * kTTWarps + wid;
    if (item >= nunits) return;
    const int it = units[item].x, jt = units[item].y;
    const int sys = b.tile_sys[it];
    const int t0 = b.tile_off[sys];
    const int as = b.atom_off[sys], ae = b.atom_off[sys + 1];
    const int ia0 = as + kTile * (it - t0), ja0 = as + kTile * (jt - t0);
    const int ni = min(kTile, ae - ia0), nj = min(kTile, ae - ja0);
    const bool diag = it == jt;
    double* oi = unit_i + ((size_t)item * kTile + lane) * kUnitI;
    const int st0 = diag ? 1 : 0, st1 = diag ? 16 : 31;
    const int mf = (lane + st1 + 1) & 31;
    double* oj = unit_j + ((size_t)item * kTile + mf) * kUnitJ;
    if (!store_ok[item]) {
        oi[0] = 0.0; oi[1] = 0.0; oi[2] = 0.0;
        oj[0] = 0.0; oj[1] = 0.0; oj[2] = 0.0;
        return;
    }
    const double dei = lane < ni ? w.dEdcn[ia0 + lane] : 0.0;
    sde[wid][lane] = lane < nj ? w.dEdcn[ja0 + lane] : 0.0;
    __syncwarp();
    double gx = 0, gy = 0, gz = 0, jx = 0, jy = 0, jz = 0;
    for (int st = st0; st <= st1; st++) {
        const int m = (lane + st) & 31;
        const R* in = store + ((size_t)item * kTile + st) * kCnStore * kTile + lane;
        const double dsum = dei + sde[wid][m];
        const double sx = double(in[0]) * dsum, sy = double(in[kTile]) * dsum, sz = double(in[2 * kTile]) * dsum;
        gx += sx; gy += sy; gz += sz;
        jx -= sx; jy -= sy; jz -= sz;
        const int src = (lane + 1) & 31;
        jx = __shfl_sync(0xffffffffu, jx, src);
        jy = __shfl_sync(0xffffffffu, jy, src);
        jz = __shfl_sync(0xffffffffu, jz, src);
    }
    oi[0] = gx; oi[1] = gy; oi[2] = gz;
    oj[0] = jx; oj[1] = jy; oj[2] = jz;
}

// An atom's sums over the slots of the items that hold it, in a fixed order,
// one warp per atom.  Lane l adds value l % VI of the atom's i slots (items
// l / VI, l / VI + 32 / VI, ...) and value l % VJ of its j slots, VI and VJ
// the powers of two >= KI and KJ, so that a warp load reads a few contiguous
// slot rows; the i slots of an atom are the items of the units (tl, jt <= tl),
// consecutive, its j slots those of the units (it >= tl, tl).  The j total of
// value m is added to i value JOFF + m; lanes 0 .. KI - 1 return the totals.
template <int KI, int KJ, int JOFF, int SJ = kUnitJ>
__device__ __forceinline__ double tt_gather_atom(long long base, int tl, int nt, int sl, int split,
                                                 const double* unit_i, const double* unit_j, int lane)
{
    constexpr int VI = KI <= 1 ? 1 : KI <= 2 ? 2 : KI <= 4 ? 4 : KI <= 8 ? 8 : 16;
    constexpr int VJ = KJ <= 1 ? 1 : KJ <= 2 ? 2 : KJ <= 4 ? 4 : 8;
    const int sh = split >> 1;   // log2 of the split (1, 2 or 4)
    double si = 0.0, sj = 0.0;
    if (lane % VI < KI) {
        const long long i0 = (base + (long long)tl * (tl + 1) / 2) * split;
        const double* p = unit_i + (i0 * kTile + sl) * kUnitI + lane % VI;
        const int ni = (tl + 1) * split;
#pragma unroll 8
        for (int q = lane / VI; q < ni; q += 32 / VI) si += p[(long long)q * (kTile * kUnitI)];
    }
#pragma unroll
    for (int o = VI; o < 32; o <<= 1) si += __shfl_xor_sync(0xffffffffu, si, o);
    if (lane % VJ < KJ) {
        const int nj = (nt - tl) * split;
#pragma unroll 8
        for (int q = lane / VJ; q < nj; q += 32 / VJ) {
            const int it = tl + (q >> sh);
            const long long item = (base + (long long)it * (it + 1) / 2 + tl) * split + (q & (split - 1));
            sj += unit_j[(item * kTile + sl) * SJ + lane % VJ];
        }
    }
#pragma unroll
    for (int o = VJ; o < 32; o <<= 1) sj += __shfl_xor_sync(0xffffffffu, sj, o);
    const int m = lane - JOFF;
    const double add = __shfl_sync(0xffffffffu, sj, m & (VJ - 1));
    if (m >= 0 && m < KJ) si += add;
    return si;
}

// Per-atom sums of the two-body unit slots: energy, dE/dCN, gradient,
// virial and parameter derivatives (lanes 0 .. 14 of tt_gather_atom).
__global__ void k_unit_gather(Batch b, Config c, const int* unit_base, int split, const double* unit_i,
                              const double* unit_j, Work w)
{
    pdl_wait();
    const int lane = threadIdx.x & 31;
    const int a = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (a >= b.natoms) return;
    const int sys = b.sys_of_atom[a];
    const int as = b.atom_off[sys];
    const int t0 = b.tile_off[sys], t1 = b.tile_off[sys + 1];
    const int tl = (a - as) / kTile;              // tile of a, local to the system
    const int sl = (a - as) % kTile;              // slot lane
    const double v = tt_gather_atom<kUnitI, kUnitJ, 1>(unit_base[sys], tl, t1 - t0, sl, split, unit_i, unit_j, lane);
    if (lane == 0) w.e_atom[a] = v;
    else if (lane == 1) { if (w.dEdcn) w.dEdcn[a] = v; }
    else if (lane < 5) { if (c.grad) w.grad[3 * a + lane - 2] = v; }
    else if (lane < 5 + kSigma) { if (c.grad) w.sig_atom[kSigma * a + lane - 5] = v; }
    else if (lane < kUnitI) { if (c.param_grad && w.pg_atom) w.pg_atom[kParamGrad * a + lane - 11] = v; }
}

// Coordination number (CHAIN = false, ncoord.f90:86-144) or its chain rule
// (CHAIN = true, ncoord.f90:152-228) over the tile-pair units with the CN
// lattice points.  Slots: CN: i [cn], j [cn]; chain: i [g(3), sigma(6)],
// j [g(3)].
// MODE 0: coordination numbers; 1: CN chain rule; 2: coordination numbers
// and, per (i, j) of the item, the translation sum of the chain rule's
// countd = dcf v / r (ncoord.f90:198-206) into `store`, for
// k_cn_chain_stored (systems of one translation chunk only), and per atom
// the sum of countd v^T over all its pairs and translations.  The chain
// rule's virial is sum over pairs of (dE/dCN_i + dE/dCN_j) countd v^T, and
// countd v^T is the same seen from i and from j, so it equals
// sum_i dE/dCN_i S_i with S_i = sum_(j, T) countd v^T (the j = i pairs of
// the T != 0 images once): six values per atom instead of six per pair.
// Slots of MODE 2: i [cn, S(6)], j in unit_i slots kCnSigJ .. [cn, S(6)].
template <class R, int MODE>
__device__ __forceinline__ void cn_tt(const Batch& b, const Species& s, const Config& c, const Partition& p,
                                      const Work& w, const int2* units, int nunits, int split, double* unit_i,
                                      double* unit_j, R* store, unsigned char* store_ok)
{
    pdl_wait();
    constexpr bool CHAIN = MODE == 1, STORE = MODE == 2;
    constexpr int NJ = STORE ? 7 : 3;
    using V = typename T4<R>::type;
    __shared__ V sth[kTTWarps][kTTChunk];
    __shared__ V stl[kTTWarps][kTTChunk];
    // FP64 j sums of the partner lanes: CN [cn], chain rule [g(3)], CN with
    // stored sums [cn, S(6)]
    __shared__ double sjs[kTTWarps][NJ][32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int item = blockIdx.x * kTTWarps + wid;
    if (item >= nunits * split) return;
    const int u = item / split, sub = item % split;
    const int splitJ = tt_split_j(split), splitT = split / splitJ;
    const int jh = sub % splitJ, th = sub / splitJ;
    const int jslots = kTile / splitJ;
    const int it = units[u].x, jt = units[u].y;
    const int sys = b.tile_sys[it];
    const int t0 = b.tile_off[sys];
    const int as = b.atom_off[sys], ae = b.atom_off[sys + 1];
    const int ia0 = as + kTile * (it - t0), ja0 = as + kTile * (jt - t0);
    const int ni = min(kTile, ae - ia0), nj = min(kTile, ae - ja0);
    const bool diag = it == jt;
    const bool ivalid = lane < ni;
    const int ic = ivalid ? ia0 + lane : ia0;
    const int li = b.local[ic];
    const double rci = s.rcov[b.sp[ic]];
    const double dei = CHAIN ? w.dEdcn[ic] : 0.0;
    const double xi = b.x[ic], yi = b.y[ic], zi = b.z[ic];
    R hix, hiy, hiz, lix = R(0), liy = R(0), liz = R(0);
    if constexpr (sizeof(R) == 8) { hix = xi; hiy = yi; hiz = zi; }
    else {
        hix = __double2float_rn(xi); lix = __double2float_rn(xi - (double)hix);
        hiy = __double2float_rn(yi); liy = __double2float_rn(yi - (double)hiy);
        hiz = __double2float_rn(zi); liz = __double2float_rn(zi - (double)hiz);
    }
    const int tt0 = b.img_off[kImgCN * (b.nsys + 1) + sys], tt1 = b.img_off[kImgCN * (b.nsys + 1) + sys + 1];
    const double4 ci = b.tiles[it], cj = b.tiles[jt];
    const double lim = c.cut_cn + ci.w + cj.w + 1.0e-6 * c.cut_cn + 1.0e-6;
    const double limj = c.cut_cn + ci.w + 1.0e-6 * c.cut_cn + 1.0e-6;
    const double dcx = ci.x - cj.x, dcy = ci.y - cj.y, dcz = ci.z - cj.z;
    const R cut2 = R(c.cut_cn * c.cut_cn);
    double (*sj)[32] = sjs[wid];
    for (int v = 0; v < NJ; v++) sj[v][lane] = 0.0;
    __syncwarp();
    // i sums: CN: a0 = cn; chain: a1..a3 gradient, a4..a8 virial xx yy zz xy xz, a0 virial yz;
    // stored sums: a1..a6 S xx yy zz xy xz yz (FP64 per partner);
    // partials in R over the partners of one translation chunk
    double a0 = 0, a1 = 0, a2 = 0, a3 = 0, a4 = 0, a5 = 0, a6 = 0, a7 = 0, a8 = 0;
    R t0_ = R(0), t1_ = R(0), t2_ = R(0), t3_ = R(0), t4_ = R(0), t5_ = R(0), t6_ = R(0), t7_ = R(0), t8_ = R(0);
    unsigned nterm = 0;
    bool ran = false;          // STORE: this item evaluated its (single) chunk
    auto flush = [&]() {
        a0 += double(t0_); t0_ = R(0);
        if (CHAIN) {
            a1 += double(t1_); a2 += double(t2_); a3 += double(t3_); a4 += double(t4_); a5 += double(t5_);
            a6 += double(t6_); a7 += double(t7_); a8 += double(t8_);
            t1_ = t2_ = t3_ = t4_ = t5_ = t6_ = t7_ = t8_ = R(0);
        }
    };
    for (int tc = tt0; tc < tt1; tc += kTTChunk) {
        const int nt = min(kTTChunk, tt1 - tc);
        const int nreach = tt_reach<V>(b.img, tc, nt, dcx, dcy, dcz, lim, lane, sth[wid], stl[wid]);
        if (nreach == 0) continue;
        const int qpart = (nreach + splitT - 1) / splitT;
        const int qbeg = th * qpart, qend = min(nreach, qbeg + qpart);
        if (qbeg >= qend) continue;
        const int jl0 = jh * jslots, jl1 = min(nj, jl0 + jslots);
        ran = true;
        for (int jl = jl0; jl < jl1; jl++) {
            const int j = ja0 + jl;
            const bool self = diag && jl == lane;
            bool valid = ivalid && (!diag || jl <= lane);
            if (valid && c.cn_partitioned && p.nparts > 1) valid = tt_owns(p, li, b.local[j]);
            if (!__any_sync(0xffffffffu, valid)) continue;
            const double xj = b.x[j], yj = b.y[j], zj = b.z[j];
            R dhx, dhy, dhz, dlx = R(0), dly = R(0), dlz = R(0);
            if constexpr (sizeof(R) == 8) { dhx = xi - xj; dhy = yi - yj; dhz = zi - zj; }
            else {
                const float4 hj = b.xhi[j], lj4 = b.xlo[j];
                dhx = hix - hj.x; dhy = hiy - hj.y; dhz = hiz - hj.z;
                dlx = lix - lj4.x; dly = liy - lj4.y; dlz = liz - lj4.z;
            }
            const R rc = R(rci + s.rcov[b.sp[j]]);
            // chain rule weight of the pair: dE/dCN_i + dE/dCN_j, or dE/dCN_i for j = i (ncoord.f90:205-213)
            const R dsum = CHAIN ? R(dei + w.dEdcn[j]) : R(0);
            const R dsig = CHAIN ? (self ? R(dei) : dsum) : R(0);
            // a lane outside the pair list accepts no term
            const R cut2v = valid ? cut2 : R(-1);
            // sums over the translations of this (i, j); the pair weights
            // dE/dCN_i + dE/dCN_j do not depend on T and multiply them afterwards
            R sc = R(0), scx = R(0), scy = R(0), scz = R(0);
            R sxx = R(0), syy = R(0), szz = R(0), sxy = R(0), sxz = R(0), syz = R(0);
            // One (i, j, T) term without branches: a term outside the cutoff
            // (or the T = 0 self pair) is evaluated at r^2 = 1 and adds zeros (tt_geo).
            auto geo = [&](int q, bool on) {
                return tt_geo<R, V>(sth[wid], stl[wid], q, dhx, dhy, dhz, dlx, dly, dlz, cut2v, R(1.0e-12), on);
            };
            auto term = [&](const TTGeo<R>& g) {
                const R vx = g.vx, vy = g.vy, vz = g.vz, r2 = g.r2;
                const bool ok = g.ok;
                nterm += ok ? 1u : 0u;
                if (STORE || CHAIN) {
                    // the count and the chain rule's countd of the same term (ncoord.f90:198-206)
                    R cf, f;
                    if constexpr (sizeof(R) == 8) {
                        const R r1 = sqrt(r2);
                        cf = R(1) / (R(1) + exp(-R(kKcnTT) * (rc / r1 - R(1))));
                        f = -cf * (R(1) - cf) * R(kKcnTT) * rc / r2 / r1;
                    } else {
                        const R ir = rsqrtf(r2);
                        cf = __fdividef(1.0f, 1.0f + expf(-R(kKcnTT) * (rc * ir - R(1))));
                        f = -cf * (R(1) - cf) * R(kKcnTT) * rc * (ir * ir * ir);
                    }
                    if (STORE) sc += ok ? cf : R(0);
                    f = ok ? f : R(0);
                    const R cx = f * vx, cy = f * vy, cz = f * vz;   // countd
                    scx += cx; scy += cy; scz += cz;
                    sxx += cx * vx; syy += cy * vy; szz += cz * vz;
                    sxy += cx * vy; sxz += cx * vz; syz += cy * vz;
                } else {
                    R cf;
                    if constexpr (sizeof(R) == 8) cf = R(1) / (R(1) + exp(-R(kKcnTT) * (rc / sqrt(r2) - R(1))));
                    else cf = __fdividef(1.0f, 1.0f + expf(-R(kKcnTT) * (rc * rsqrtf(r2) - R(1))));
                    sc += ok ? cf : R(0);
                }
            };
            unsigned jm[kJMaskWords];
            const int nw = tt_jmask<V>(sth[wid], stl[wid], qbeg, qend, ci, xj, yj, zj, limj, lane, jm);
#pragma unroll
            for (int h = 0; h < kJMaskWords; h++) {
                if (h >= nw) break;
                const int qh = qbeg + 32 * h - 1;
                for (unsigned mm = jm[h]; mm;) {
                    const int qa = qh + __ffs(mm);
                    mm &= mm - 1;
                    if constexpr (kPairStep<R>) {
                        const bool two = mm != 0u;
                        const int qb = two ? qh + __ffs(mm) : qa;
                        mm &= mm - 1;
                        term(geo(qa, true));
                        term(geo(qb, two));
                    } else {
                        const TTGeo<R> ga = geo(qa, true);
                        if (ga.ok) term(ga);
                    }
                }
            }
            if (STORE) {
                R* out = store + ((size_t)item * jslots + (jl - jl0)) * kCnStore * kTile + lane;
                const R vals[kCnStore] = {scx, scy, scz};
#pragma unroll
                for (int v = 0; v < kCnStore; v++) out[v * kTile] = vals[v];
                t0_ += sc;
                a1 += double(sxx); a2 += double(syy); a3 += double(szz);
                a4 += double(sxy); a5 += double(sxz); a6 += double(syz);
                // the column atom's cn and S (the j = i image pairs count once, on the row side)
                const R z0 = wsum4_tt<R>(self ? R(0) : sc, self ? R(0) : sxx, self ? R(0) : syy,
                                         self ? R(0) : szz, lane);
                const R z1 = wsum4_tt<R>(self ? R(0) : sxy, self ? R(0) : sxz, self ? R(0) : syz, R(0), lane);
                if ((lane & 7) == 0) {
                    sj[lane >> 3][jl] += double(z0);
                    if (lane < 24) sj[4 + (lane >> 3)][jl] += double(z1);
                }
            } else if (!CHAIN) {
                t0_ += sc;
                const R z = wsum_tt<R>(self ? R(0) : sc);
                if (lane == 0) sj[0][jl] += double(z);
            } else {
                R j0 = R(0), j1 = R(0), j2 = R(0);
                if (!self) {
                    t1_ += scx * dsum; t2_ += scy * dsum; t3_ += scz * dsum;
                    j0 = -scx * dsum; j1 = -scy * dsum; j2 = -scz * dsum;
                }
                t4_ += sxx * dsig; t5_ += syy * dsig; t6_ += szz * dsig;
                t7_ += sxy * dsig; t8_ += sxz * dsig; t0_ += syz * dsig;
                // lane 8v holds the warp sum of value v
                const R z = wsum4_tt<R>(j0, j1, j2, R(0), lane);
                if ((lane & 7) == 0 && lane < 24) sj[lane >> 3][jl] += double(z);
            }
        }
        flush();
    }
    __syncwarp();
    double* oi = unit_i + ((size_t)item * kTile + lane) * kUnitI;
    double* oj = unit_j + ((size_t)item * kTile + lane) * kUnitJ;
    if (STORE) {
        oi[0] = a0;
        oi[1] = a1; oi[2] = a2; oi[3] = a3; oi[4] = a4; oi[5] = a5; oi[6] = a6;
#pragma unroll
        for (int v = 0; v < 7; v++) oi[kCnSigJ + v] = sj[v][lane];
    } else if (!CHAIN) {
        oi[0] = a0;
        oj[0] = sj[0][lane];
    } else {
        // g(3), sigma xx yy zz xy xz yz
        oi[0] = a1; oi[1] = a2; oi[2] = a3;
        oi[3] = a4; oi[4] = a5; oi[5] = a6; oi[6] = a7; oi[7] = a8; oi[8] = a0;
        oj[0] = sj[0][lane]; oj[1] = sj[1][lane]; oj[2] = sj[2][lane];
    }
    if (STORE && lane == 0) store_ok[item] = ran ? 1 : 0;
    if (!CHAIN && w.counts) {
        unsigned long long n = nterm;
        for (int off = 16; off > 0; off >>= 1) n += __shfl_xor_sync(0xffffffffu, n, off);
        if (lane == 0) atomicAdd(w.counts + 2, n);
    }
}

template <class R, int MODE>
__global__ void __launch_bounds__(kTTThreads)
k_cn_tt(Batch b, Species s, Config c, Partition p, Work w, const int2* units, int nunits, int split, double* unit_i,
        double* unit_j, R* store, unsigned char* store_ok)
{
    cn_tt<R, MODE>(b, s, c, p, w, units, nunits, split, unit_i, unit_j, store, store_ok);
}

// The FP64 stored-sum pass held to 128 registers: four blocks per SM instead
// of three (a few bytes of spills; 142 registers unbounded).
__global__ void __launch_bounds__(kTTThreads, 4)
k_cn_tt_store64(Batch b, Species s, Config c, Partition p, Work w, const int2* units, int nunits, int split,
                double* unit_i, double* unit_j, double* store, unsigned char* store_ok)
{
    cn_tt<double, 2>(b, s, c, p, w, units, nunits, split, unit_i, unit_j, store, store_ok);
}

// CN chain rule gradient from the sums k_cn_tt<R, 2> stored: per (i, j) of
// the item the weight dE/dCN_i + dE/dCN_j times the stored countd sums
// (ncoord.f90:205-209); slots i [g(3)], j [g(3)].  The virial follows per
// atom from the S sums of the CN pass (k_cn_gather<true, true>).
template <class R>
__global__ void __launch_bounds__(kTTThreads)
k_cn_chain_stored(Batch b, Config c, Partition p, Work w, const int2* units, int nunits, int split, const R* store,
                  const unsigned char* store_ok, double* unit_i, double* unit_j)
{
    pdl_wait();
    __shared__ double sjs[kTTWarps][3][32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int item = blockIdx.x * kTTWarps + wid;
    if (item >= nunits * split) return;
    const int u = item / split, sub = item % split;
    const int splitJ = tt_split_j(split);
    const int jh = sub % splitJ;
    const int jslots = kTile / splitJ;
    const int it = units[u].x, jt = units[u].y;
    const int sys = b.tile_sys[it];
    const int t0 = b.tile_off[sys];
    const int as = b.atom_off[sys], ae = b.atom_off[sys + 1];
    const int ia0 = as + kTile * (it - t0), ja0 = as + kTile * (jt - t0);
    const int ni = min(kTile, ae - ia0), nj = min(kTile, ae - ja0);
    const bool diag = it == jt;
    const bool ivalid = lane < ni;
    const int ic = ivalid ? ia0 + lane : ia0;
    const int li = b.local[ic];
    const double dei = w.dEdcn[ic];
    double (*sj)[32] = sjs[wid];
    for (int v = 0; v < 3; v++) sj[v][lane] = 0.0;
    __syncwarp();
    double g[3] = {0, 0, 0};
    if (store_ok[item]) {
        const int jl0 = jh * jslots, jl1 = min(nj, jl0 + jslots);
        // the sums of NQ partners are loaded together (memory-level parallelism);
        // sums of a partner that no lane of the item took were not stored and
        // are loaded but not used
        constexpr int NQ = sizeof(R) == 4 ? 8 : 4;
        for (int jg = jl0; jg < jl1; jg += NQ) {
            R sv[NQ][kCnStore];
#pragma unroll
            for (int q = 0; q < NQ; q++) {
                const R* in = store + ((size_t)item * jslots + min(jg + q, jl1 - 1) - jl0) * kCnStore * kTile + lane;
#pragma unroll
                for (int v = 0; v < kCnStore; v++) sv[q][v] = in[v * kTile];
            }
#pragma unroll
            for (int q = 0; q < NQ; q++) {
                const int jl = jg + q;
                if (jl >= jl1) break;
                const int j = ja0 + jl;
                const bool self = diag && jl == lane;
                bool valid = ivalid && (!diag || jl <= lane);
                if (valid && c.cn_partitioned && p.nparts > 1) valid = tt_owns(p, li, b.local[j]);
                if (!__any_sync(0xffffffffu, valid)) continue;
                const double dsum = dei + w.dEdcn[j];
                double j0 = 0.0, j1 = 0.0, j2 = 0.0;
                if (!self) {
                    const double sx = double(sv[q][0]), sy = double(sv[q][1]), sz = double(sv[q][2]);
                    g[0] += sx * dsum; g[1] += sy * dsum; g[2] += sz * dsum;
                    j0 = -sx * dsum; j1 = -sy * dsum; j2 = -sz * dsum;
                }
                // lane 8v holds the warp sum of value v
                const double z = wsum4_tt<double>(j0, j1, j2, 0.0, lane);
                if ((lane & 7) == 0 && lane < 24) sj[lane >> 3][jl] += z;
            }
        }
    }
    __syncwarp();
    double* oi = unit_i + ((size_t)item * kTile + lane) * kUnitI;
    double* oj = unit_j + ((size_t)item * kTile + lane) * kUnitJ;
    oi[0] = g[0]; oi[1] = g[1]; oi[2] = g[2];
    oj[0] = sj[0][lane]; oj[1] = sj[1][lane]; oj[2] = sj[2][lane];
}

// Gather of the CN (assign) or chain-rule (add to gradient and virial) slots,
// one warp per atom, in the fixed order of tt_gather_atom.  STORED: the slots
// of the stored-sum passes, with the atom's S sums (CN) and its chain-rule
// virial dE/dCN_i S_i (chain rule).
template <bool CHAIN, bool STORED>
__global__ void k_cn_gather(Batch b, const int* unit_base, int split, const double* unit_i, const double* unit_j,
                            Work w)
{
    pdl_wait();
    const int lane = threadIdx.x & 31;
    const int a = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (a >= b.natoms) return;
    const int sys = b.sys_of_atom[a];
    const int as = b.atom_off[sys];
    const int t0 = b.tile_off[sys], t1 = b.tile_off[sys + 1];
    const int tl = (a - as) / kTile, sl = (a - as) % kTile;
    if (!CHAIN && STORED) {
        const double v = tt_gather_atom<7, 7, 0, kUnitI>(unit_base[sys], tl, t1 - t0, sl, split, unit_i,
                                                         unit_i + kCnSigJ, lane);
        if (lane == 0) w.cn[a] = v;
        else if (lane < 7) w.cn_sig[kSigma * a + lane - 1] = v;
    } else if (!CHAIN) {
        const double v = tt_gather_atom<1, 1, 0>(unit_base[sys], tl, t1 - t0, sl, split, unit_i, unit_j, lane);
        if (lane == 0) w.cn[a] = v;
    } else if (STORED) {
        const double v = tt_gather_atom<3, 3, 0>(unit_base[sys], tl, t1 - t0, sl, split, unit_i, unit_j, lane);
        if (lane < 3) w.grad[3 * a + lane] += v;
        else if (lane < 9) w.sig_atom[kSigma * a + lane - 3] += w.dEdcn[a] * w.cn_sig[kSigma * a + lane - 3];
    } else {
        // g(3), sigma(6); j slots g(3)
        const double v = tt_gather_atom<9, 3, 0>(unit_base[sys], tl, t1 - t0, sl, split, unit_i, unit_j, lane);
        if (lane < 3) w.grad[3 * a + lane] += v;
        else if (lane < 9) w.sig_atom[kSigma * a + lane - 3] += v;
    }
}


// After the CN sweep, one warp per atom: the CN from the unit slots, the
// Gaussian reference weights and their CN derivative with the reference's
// NaN/Inf fallback (weight_references, model.f90:201-324; FP64, the
// arithmetic of k_weights: lane r takes reference r, the sums run in
// reference order) and, when UV is given, the atom's species vectors for
// the two-body sweep (the entries of k_species_vectors).
template <class R>
__global__ void k_cn_weights(Batch b, Species s, Config c, const int* unit_base, int split, const double* unit_i,
                             const double* unit_j, Work w, R* UV, bool stored)
{
    pdl_wait();
    const int lane = threadIdx.x & 31;
    const int a = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (a >= b.natoms) return;
    const int sys = b.sys_of_atom[a];
    const int as = b.atom_off[sys];
    const int t0 = b.tile_off[sys], t1 = b.tile_off[sys + 1];
    const int tl = (a - as) / kTile, sl = (a - as) % kTile;
    double cn;
    if (stored) {
        // the CN and the atom's S sums of the stored-sum pass
        const double v = tt_gather_atom<7, 7, 0, kUnitI>(unit_base[sys], tl, t1 - t0, sl, split, unit_i,
                                                         unit_i + kCnSigJ, lane);
        if (lane >= 1 && lane < 7) w.cn_sig[kSigma * a + lane - 1] = v;
        cn = __shfl_sync(0xffffffffu, v, 0);
    } else {
        cn = __shfl_sync(0xffffffffu,
                         tt_gather_atom<1, 1, 0>(unit_base[sys], tl, t1 - t0, sl, split, unit_i, unit_j, lane), 0);
    }
    if (lane == 0) w.cn[a] = cn;
    atom_weights<R>(b, s, c, w, a, cn, lane, UV);
}

template <class R, int DAMP, bool GRAD, bool PG>
void launch_tt(const Batch& b, const Species& s, const Damp& d, const Config& c, const Partition& p, const Work& w,
               const PairUnits& pu, cudaStream_t stream)
{
    const int blocks = (pu.nunits * pu.split + kTTWarps - 1) / kTTWarps;
    const bool smooth = c.width2 > 0.0 && c.width2 < c.cut2;
#define D3_TT(SM, CO)                                                                                   \
    launch_pdl(k_two_body_tt<R, DAMP, GRAD, PG, SM, CO>, dim3(blocks), dim3(kTTThreads), 0, stream, \
        b, s, d, c, p, w, pu.units, pu.nunits, pu.split, (const R*)pu.U, pu.unit_i, pu.unit_j)
    if (w.counts) {
        if (smooth) D3_TT(true, true);
        else D3_TT(false, true);
    } else {
        if (smooth) D3_TT(true, false);
        else D3_TT(false, false);
    }
#undef D3_TT
}

// the families without damping-parameter derivatives (the engine refuses
// them for those)
template <class R, int DAMP>
void launch_tt_family(const Batch& b, const Species& s, const Damp& d, const Config& c, const Partition& p,
                      const Work& w, const PairUnits& pu, cudaStream_t stream)
{
    if (c.grad) launch_tt<R, DAMP, true, false>(b, s, d, c, p, w, pu, stream);
    else launch_tt<R, DAMP, false, false>(b, s, d, c, p, w, pu, stream);
}

template <class R, int DAMP>
void launch_tt_flags(const Batch& b, const Species& s, const Damp& d, const Config& c, const Partition& p,
                     const Work& w, const PairUnits& pu, cudaStream_t stream)
{
    if (c.grad) {
        if (c.param_grad) launch_tt<R, DAMP, true, true>(b, s, d, c, p, w, pu, stream);
        else launch_tt<R, DAMP, true, false>(b, s, d, c, p, w, pu, stream);
    } else {
        if (c.param_grad) launch_tt<R, DAMP, false, true>(b, s, d, c, p, w, pu, stream);
        else launch_tt<R, DAMP, false, false>(b, s, d, c, p, w, pu, stream);
    }
}

}  // namespace

void launch_cn_units(const Batch& b, const Species& s, const Config& c, const Partition& p, const Work& w,
                     const PairUnits& pu, bool chain, cudaStream_t stream, bool weights, void* uv)
{
    if (b.natoms <= 0) return;
    const int blocks = (pu.nunits * pu.split + kTTWarps - 1) / kTTWarps;
    const bool stored = pu.cn_store != nullptr;
#define D3_CN(R, MODE)                                                                                     \
    launch_pdl(k_cn_tt<R, MODE>, dim3(blocks), dim3(kTTThreads), 0, stream, b, s, c, p, w, pu.units, pu.nunits, pu.split,     \
                                                        pu.unit_i, pu.unit_j, (R*)pu.cn_store, pu.cn_store_ok)
    // molecules: the diagonal walk (CN with stored sums or alone, chain rule from the stored sums)
    const bool rot = pu.single_image && pu.split == 1 && p.nparts <= 1 && !c.cn_partitioned && !w.counts &&
                     (stored || !chain);
    if (rot && pu.nunits > 0) {
        const dim3 grid(blocks), block(kTTThreads);
        if (chain) {
            if (c.mixed)
                launch_pdl(k_cn_chain_rot<float>, grid, block, 0, stream, b, w, pu.units, pu.nunits,
                           (const float*)pu.cn_store, pu.cn_store_ok, pu.unit_i, pu.unit_j);
            else
                launch_pdl(k_cn_chain_rot<double>, grid, block, 0, stream, b, w, pu.units, pu.nunits,
                           (const double*)pu.cn_store, pu.cn_store_ok, pu.unit_i, pu.unit_j);
        } else if (stored) {
            if (c.mixed)
                launch_pdl(k_cn_rot<float, true>, grid, block, 0, stream, b, s, c, w, pu.units, pu.nunits, pu.unit_i,
                           pu.unit_j, (float*)pu.cn_store, pu.cn_store_ok);
            else
                launch_pdl(k_cn_rot<double, true>, grid, block, 0, stream, b, s, c, w, pu.units, pu.nunits, pu.unit_i,
                           pu.unit_j, (double*)pu.cn_store, pu.cn_store_ok);
        } else {
            if (c.mixed)
                launch_pdl(k_cn_rot<float, false>, grid, block, 0, stream, b, s, c, w, pu.units, pu.nunits, pu.unit_i,
                           pu.unit_j, (float*)nullptr, pu.cn_store_ok);
            else
                launch_pdl(k_cn_rot<double, false>, grid, block, 0, stream, b, s, c, w, pu.units, pu.nunits,
                           pu.unit_i, pu.unit_j, (double*)nullptr, pu.cn_store_ok);
        }
    } else if (pu.nunits > 0) {
        if (chain && stored) {
            if (c.mixed)
                launch_pdl(k_cn_chain_stored<float>, dim3(blocks), dim3(kTTThreads), 0, stream, b, c, p, w, pu.units, pu.nunits, pu.split, (const float*)pu.cn_store, pu.cn_store_ok, pu.unit_i,
                    pu.unit_j);
            else
                launch_pdl(k_cn_chain_stored<double>, dim3(blocks), dim3(kTTThreads), 0, stream, b, c, p, w, pu.units, pu.nunits, pu.split, (const double*)pu.cn_store, pu.cn_store_ok, pu.unit_i,
                    pu.unit_j);
        } else if (chain) {
            if (c.mixed) D3_CN(float, 1);
            else D3_CN(double, 1);
        } else if (stored) {
            if (c.mixed) D3_CN(float, 2);
            else
                launch_pdl(k_cn_tt_store64, dim3(blocks), dim3(kTTThreads), 0, stream, b, s, c, p, w, pu.units,
                           pu.nunits, pu.split, pu.unit_i, pu.unit_j, (double*)pu.cn_store, pu.cn_store_ok);
        } else {
            if (c.mixed) D3_CN(float, 0);
            else D3_CN(double, 0);
        }
    }
#undef D3_CN
    const unsigned gb = (unsigned)((b.natoms + 7) / 8);
#define D3_GATHER(CH, ST) \
    launch_pdl(k_cn_gather<CH, ST>, dim3(gb), dim3(256), 0, stream, b, pu.unit_base, pu.split, pu.unit_i, pu.unit_j, w)
    if (chain) {
        if (stored) D3_GATHER(true, true);
        else D3_GATHER(true, false);
    } else if (!weights) {
        if (stored) D3_GATHER(false, true);
        else D3_GATHER(false, false);
    } else if (c.mixed)
        launch_pdl(k_cn_weights<float>, dim3(gb), dim3(256), 0, stream, b, s, c, pu.unit_base, pu.split, pu.unit_i, pu.unit_j, w,
                                                     (float*)uv, stored);
    else
        launch_pdl(k_cn_weights<double>, dim3(gb), dim3(256), 0, stream, b, s, c, pu.unit_base, pu.split, pu.unit_i, pu.unit_j, w,
                                                      (double*)uv, stored);
#undef D3_GATHER
}

size_t cn_store_bytes(const PairUnits& pu, bool mixed)
{
    return (size_t)pu.nunits * pu.split * (kTile / tt_split_j(pu.split)) * kCnStore * kTile *
           (mixed ? sizeof(float) : sizeof(double));
}

size_t pair_unit_slot_doubles() { return (size_t)kSplitMax * kTile * (kUnitI + kUnitJ); }
size_t pair_unit_i_doubles() { return (size_t)kSplitMax * kTile * kUnitI; }
size_t species_vector_doubles(int natoms, int nid) { return (size_t)natoms * nid * 2 * kRefPad; }

void launch_species_vectors(const Batch& b, const Species& s, const Config& c, const Work& w, void* U,
                            cudaStream_t stream)
{
    if (b.natoms <= 0) return;
    const long long nsv = (long long)b.natoms * b.nid * kRefPad;
    if (c.mixed)
        launch_pdl(k_species_vectors<float>, dim3((unsigned)((nsv + 255) / 256)), dim3(256), 0, stream, b, s, w, (float*)U);
    else
        launch_pdl(k_species_vectors<double>, dim3((unsigned)((nsv + 255) / 256)), dim3(256), 0, stream, b, s, w, (double*)U);
}

void launch_two_body_units(const Batch& b, const Species& s, const Damp& d, const Config& c, const Partition& p,
                           const Work& w, const PairUnits& pu, cudaStream_t stream, cudaEvent_t ev_begin,
                           cudaEvent_t ev_end, bool species_ready)
{
    if (b.natoms <= 0) return;
    const long long nsv = (long long)b.natoms * b.nid * kRefPad;
    if (species_ready) {
        // k_cn_weights wrote the species vectors
    } else if (c.mixed)
        launch_pdl(k_species_vectors<float>, dim3((unsigned)((nsv + 255) / 256)), dim3(256), 0, stream, b, s, w, (float*)pu.U);
    else
        launch_pdl(k_species_vectors<double>, dim3((unsigned)((nsv + 255) / 256)), dim3(256), 0, stream, b, s, w, (double*)pu.U);
    if (ev_begin) cudaEventRecord(ev_begin, stream);
    // molecules only (one lattice point), rational or zero damping, gradient,
    // no parameter derivatives, smooth cutoff, counters or partition: the
    // diagonal walk without translation lists
    const bool smooth = c.width2 > 0.0 && c.width2 < c.cut2;
    const bool rot = pu.single_image && pu.split == 1 && c.grad && !c.param_grad && !smooth && !w.counts &&
                     p.nparts <= 1 && b.nid <= kMaxSpeciesFast && (d.kind == kRational || d.kind == kZero);
    if (rot && pu.nunits > 0) {
        const dim3 grid((pu.nunits + kTTWarps - 1) / kTTWarps), block(kTTThreads);
#define D3_ROT(R, DK) \
    launch_pdl(k_two_body_rot<R, DK>, grid, block, 0, stream, b, s, d, c, w, pu.units, pu.nunits, (const R*)pu.U, \
               pu.unit_i, pu.unit_j)
        if (d.kind == kRational) { if (c.mixed) D3_ROT(float, kRational); else D3_ROT(double, kRational); }
        else { if (c.mixed) D3_ROT(float, kZero); else D3_ROT(double, kZero); }
#undef D3_ROT
    } else if (pu.nunits > 0) {
        switch (d.kind) {
        case kRational:
            if (c.mixed) launch_tt_flags<float, kRational>(b, s, d, c, p, w, pu, stream);
            else launch_tt_flags<double, kRational>(b, s, d, c, p, w, pu, stream);
            break;
        case kZero:
            if (c.mixed) launch_tt_flags<float, kZero>(b, s, d, c, p, w, pu, stream);
            else launch_tt_flags<double, kZero>(b, s, d, c, p, w, pu, stream);
            break;
        case kMZero:
            if (c.mixed) launch_tt_family<float, kMZero>(b, s, d, c, p, w, pu, stream);
            else launch_tt_family<double, kMZero>(b, s, d, c, p, w, pu, stream);
            break;
        case kOptimizedPower:
            if (c.mixed) launch_tt_family<float, kOptimizedPower>(b, s, d, c, p, w, pu, stream);
            else launch_tt_family<double, kOptimizedPower>(b, s, d, c, p, w, pu, stream);
            break;
        case kCSO:
            if (c.mixed) launch_tt_family<float, kCSO>(b, s, d, c, p, w, pu, stream);
            else launch_tt_family<double, kCSO>(b, s, d, c, p, w, pu, stream);
            break;
        default:
            if (c.mixed) launch_tt_family<float, kZDamping>(b, s, d, c, p, w, pu, stream);
            else launch_tt_family<double, kZDamping>(b, s, d, c, p, w, pu, stream);
            break;
        }
    }
    if (ev_end) cudaEventRecord(ev_end, stream);
    launch_pdl(k_unit_gather, dim3((b.natoms + 7) / 8), dim3(256), 0, stream, b, c, pu.unit_base, pu.split, pu.unit_i, pu.unit_j, w);
}

}  // namespace d3
