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
//   k_nbr_fill      entries image by image (for each translation T the atoms
//                   j <= i in spatial order): vector x_j + T - x_i and r^2
//   k_triples       persistent blocks take roots from a queue (largest lists
//                   first); the warps sweep 32 x 32 tiles of (entry, entry)
//                   pairs in the rounds of a round-robin schedule (disjoint
//                   tiles per round), walking each tile along its diagonals
//                   with the column sums travelling between the lanes, and
//                   skip the steps in which no candidate is inside the cutoff
//                   (the image-by-image order keeps tiles compact).  Per-entry
//                   sums (scalar pair factor S, jk-gradient G, dE/dCN share D)
//                   are updated in a fixed order; at the end of the root the
//                   force and dE/dCN share of every entry's atom, and the
//                   root's own, are added to per-atom fixed-point accumulators
//                   (integer additions, so their order does not matter).
//   k_atm_fixed     the accumulators into the FP64 gradient and dE/dCN: the
//                   result is bit-reproducible in both forms.

#include <cub/cub.cuh>

#include <algorithm>

#include <cfloat>
#include <cstdint>

#include "d3_device.cuh"
#include "d3_atm_common.cuh"

namespace d3 {

namespace {

constexpr int kThreadsAtm = 256; // 8 warps
// resident blocks per SM the triple kernel is compiled for (FP32 and FP64 forms)
#ifndef TRI_MINB_F
#define TRI_MINB_F 3
#endif
#ifndef TRI_MINB_D
#define TRI_MINB_D 2
#endif
constexpr int kAcc = 5;          // per-entry accumulators: S, Gx, Gy, Gz, dE/dCN of the partner

// ------------------------------------------------------------ C6 matrix ----

// {sqrt(C6_rc), dC6_rc/dCN_r / C6_rc, dC6_rc/dCN_c / C6_rc} for every ordered
// pair (r, c) of each system (get_atomic_c6, model.f90:432-461); ghosts give 0.
// The double sum over the references is taken as a dot product of r's
// weights with c's species vector for r's species, U_c[s_r][ir] =
// sum_jr C6ref(ir, jr) gw_c[jr] (and dU with dgw), accumulated in FP64.
// One warp per row r; the lanes take the columns.  The damping-radius terms
// alp3 log(r0) of the row's species pairs are computed once per row (for up
// to 32 species), the species vectors are read with vector loads.
template <class R>
__global__ void k_c6_matrix(Batch b, Species s, Work w, const R* UV, double alp3, const long long* mat_off,
                            C6Entry<R>* mat)
{
    __shared__ R slr0[8][32];
    const int lane = threadIdx.x & 31, wid = (threadIdx.x >> 5) & 7;
    const int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (r >= b.natoms) return;
    const int sys = b.sys_of_atom[r];
    const int a0 = b.atom_off[sys];
    const int n = b.atom_off[sys + 1] - a0;
    C6Entry<R>* row = mat + mat_off[sys] + (long long)(r - a0) * n;
    const int sr = b.sp[r];
    const int nr = s.nref[sr];
    const bool gr = b.ghost && b.ghost[r];
    const bool table = b.nid <= 32;
    auto lr0_of = [&](int sc) {
        const double r0 = __ldg(s.atm_r0 + sr * b.nid + sc);
        return R(alp3 * (sizeof(R) == 8 ? log(r0) : log2(r0)));
    };
    if (table && lane < b.nid) slr0[wid][lane] = lr0_of(lane);
    __syncwarp();
    const R* gw = (const R*)(sizeof(R) == 8 ? (const void*)w.gw : (const void*)w.gwf) + (size_t)r * kMaxRef;
    const R* dgw = (const R*)(sizeof(R) == 8 ? (const void*)w.dgw : (const void*)w.dgwf) + (size_t)r * kMaxRef;
    double g[kRefPad], dg[kRefPad];
#pragma unroll
    for (int ir = 0; ir < kRefPad; ir++) {
        g[ir] = ir < nr ? double(gw[ir]) : 0.0;
        dg[ir] = ir < nr ? double(dgw[ir]) : 0.0;
    }
    // the lower triangle (c <= r) and its mirror: C6 is symmetric and the entry
    // (c, r) swaps the two CN-derivative ratios (the damping radius table is
    // symmetric), so every product is formed once
    const int rl = r - a0;
    C6Entry<R>* mat_sys = mat + mat_off[sys];
    for (int cl = lane; cl <= rl; cl += 32) {
        const int c = a0 + cl;
        const int sc = b.sp[c];
        const R lr0 = table ? slr0[wid][sc] : lr0_of(sc);
        C6Entry<R> out{R(0), R(0), R(0), lr0};
        if (!(gr || (b.ghost && b.ghost[c]))) {
            // U[0..7] and dU[0..7] of atom c for species sr (padding entries are zero)
            R u[2 * kRefPad];
            const R* up = UV + ((size_t)c * b.nid + sr) * (2 * kRefPad);
            if constexpr (sizeof(R) == 4) {
#pragma unroll
                for (int q = 0; q < kRefPad / 2; q++) {
                    const float4 v = __ldg(reinterpret_cast<const float4*>(up) + q);
                    u[4 * q] = v.x; u[4 * q + 1] = v.y; u[4 * q + 2] = v.z; u[4 * q + 3] = v.w;
                }
            } else {
#pragma unroll
                for (int q = 0; q < kRefPad; q++) {
                    const double2 v = __ldg(reinterpret_cast<const double2*>(up) + q);
                    u[2 * q] = v.x; u[2 * q + 1] = v.y;
                }
            }
            if constexpr (sizeof(R) == 4) {
                // the FP32 entries of the mixed form from FP32 operands: FP32 arithmetic
                float c6 = 0.f, dr = 0.f, dc = 0.f;
#pragma unroll
                for (int ir = 0; ir < kMaxRef; ir++) {
                    c6 += float(g[ir]) * u[ir];
                    dr += float(dg[ir]) * u[ir];
                    dc += float(g[ir]) * u[kRefPad + ir];
                }
                if (c6 != 0.f) {
                    const float inv = 1.0f / c6;
                    out = C6Entry<R>{sqrtf(c6), dr * inv, dc * inv, lr0};
                }
            } else {
                double c6 = 0.0, dr = 0.0, dc = 0.0;
#pragma unroll
                for (int ir = 0; ir < kMaxRef; ir++) {
                    const double uv = double(u[ir]), du = double(u[kRefPad + ir]);
                    c6 += g[ir] * uv;
                    dr += dg[ir] * uv;
                    dc += g[ir] * du;
                }
                if (c6 != 0.0) {
                    const double inv = 1.0 / c6;
                    out = C6Entry<R>{R(sqrt(c6)), R(dr * inv), R(dc * inv), lr0};
                }
            }
        }
        row[cl] = out;
        if (cl < rl) mat_sys[(long long)cl * n + rl] = C6Entry<R>{out.sc6, out.qcr, out.qrc, out.lr0};
    }
}

// --------------------------------------------------------- neighbour lists --

__device__ __forceinline__ bool in_shell(double r2, double cut2) { return !(r2 > cut2 || r2 < DBL_EPSILON); }

// |v|^2 with a fixed rounding sequence, so that the counting and the filling
// of the lists take exactly the same decisions
__device__ __forceinline__ double norm2(double x, double y, double z)
{
    return __fma_rn(z, z, __fma_rn(y, y, __dmul_rn(x, x)));
}

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
            n += in_shell(norm2(vx, vy, vz), cut2);
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

// Entries of root i, image by image: for each lattice translation T the
// atoms j <= i (in the batch's spatial order) with eps <= |x_j + T - x_i|^2
// <= cutoff^2, so that runs of consecutive entries are compact in space.
// vec = (x_j + T) - x_i as in atm.f90:718.
__global__ void k_nbr_fill(Batch b, Config c, const uint8_t* sys_skip, const long long* off, const int* cnt,
                           int* nbr_j, int* nbr_gend, double4* nbr_v, const int* guard)
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
    const long long end = off[i] + cnt[i];
    for (int t = t0; t < t1; t++) {
        const double tx = __ldg(b.img + 3 * t), ty = __ldg(b.img + 3 * t + 1), tz = __ldg(b.img + 3 * t + 2);
        for (int jb = j0; jb <= i; jb += 32) {
            const int j = jb + lane;
            const bool valid = j <= i;
            // the arithmetic of k_nbr_count, so that both accept the same entries
            // (a self image at exactly the cutoff must not be counted and then missed)
            const double dx = valid ? b.x[j] - xi : 0.0, dy = valid ? b.y[j] - yi : 0.0,
                         dz = valid ? b.z[j] - zi : 0.0;
            const double vx = dx + tx, vy = dy + ty, vz = dz + tz;
            const double r2 = norm2(vx, vy, vz);
            const bool ok = valid && in_shell(r2, cut2);
            const unsigned msk = __ballot_sync(0xffffffffu, ok);
            if (ok) {
                const long long p = pos + __popc(msk & ((1u << lane) - 1u));
                if (p < end) {
                    nbr_j[p] = j;
                    nbr_gend[p] = 0;
                    nbr_v[p] = make_double4(vx, vy, vz, r2);
                }
            }
            pos += __popc(msk);
        }
    }
    // the list holds exactly the counted entries: slots the fill did not reach
    // (which identical arithmetic rules out) become empty entries (r^2 = -1)
    for (long long q = pos + lane; q < end; q += 32) {
        nbr_j[q] = i;
        nbr_gend[q] = 0;
        nbr_v[q] = make_double4(0.0, 0.0, 0.0, -1.0);
    }
}

// Deterministic accumulation of per-atom sums from many blocks: a value is
// added as two 64-bit integers, its multiple of 2^-32 (floor) and the rest
// rounded to units of 2^-72, so that the total does not depend on the order
// of the additions.  Range +-2^31 per addition; the rest word takes up to
// 2^23 additions (each below 2^40 + 1) before it could overflow.
__device__ __forceinline__ void fixed_add(unsigned long long* acc2, double v)
{
    const double sv = v * 4294967296.0;                 // 2^32
    const double h = floor(sv);
    const long long hi = (long long)h;
    const long long lo = __double2ll_rn((sv - h) * 1099511627776.0);   // 2^40
    atomicAdd(acc2, (unsigned long long)hi);
    atomicAdd(acc2 + 1, (unsigned long long)lo);
}

__device__ __forceinline__ double fixed_value(const unsigned long long* acc2)
{
    return double((long long)acc2[0]) * 2.3283064365386963e-10 +      // 2^-32
           double((long long)acc2[1]) * 2.117582368135751e-22;        // 2^-72
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
    typename Vec4<R>::type s;   // 1/r, switch, dsw/dr / r, valid (1 or 0)
    int4 meta;                  // atom, group end, species, input index
};

// Column entries of one warp's tile pair, one array per field (rotated reads
// of the lanes hit consecutive slots).
template <class R>
struct EntryTile {
    typename Vec4<R>::type v[32], l[32], c[32], s[32];
    int4 meta[32];
};

// Entry tiles a and b of the round-robin schedule of T' (even) tiles: round r
// < T' - 1 pairs tile T' - 1 with r and (r + k) with (r - k) (mod T' - 1),
// k = 1 .. T'/2 - 1; every tile is in exactly one pair of a round.
__device__ __forceinline__ void rr_pair(int r, int k, int tp, int& a, int& b)
{
    const int q = tp - 1;
    if (k == 0) { a = q; b = r; }
    else { a = (r + k) % q; b = (r - k + q) % q; }
}

// Triple sum of the roots.  Persistent blocks take roots from a queue
// (largest lists first).  A root's entries (j <= i, T) are cut into tiles of
// 32, and every unordered pair of entries {a, b} is one candidate triple
// (i, j, k): the atom pair (j, k) is the pair of entry atoms, larger first,
// and two images of one atom stand for both orders of the reference's loop
// (atm.f90:705-733), so they count twice (triple_scale, atm.f90:954-980, of
// the atoms times 2).  The tile pairs (A, B) run in rounds of a round-robin
// schedule, in which every tile occurs in one pair, and the block waits at
// the end of each round; within a round the warps own their tiles alone, so
// the per-entry sums are updated without atomics and in a fixed order, and
// the result is bit-reproducible.  A warp walks its 32 x 32 tile pair along
// the diagonals: at step t lane l pairs row entry 32 A + l with column entry
// 32 B + (l + t) mod 32; the column's five sums move one lane down per step
// with the column, the row's stay in the lane.  The diagonal pairs (A, A)
// take steps 1..16.  Candidates are evaluated without branches (weight zero
// outside the cutoff).
template <class R, bool GRAD, bool PER, bool SMOOTH>
__global__ void __launch_bounds__(kThreadsAtm, sizeof(R) == 4 ? TRI_MINB_F : TRI_MINB_D)
k_triples(Batch b, Species sp, Damp d, Config c, Partition part, Work w, const C6Entry<R>* mat,
          const long long* mat_off, const long long* off, const int* cnt, const int* nbr_j, const int* nbr_gend,
          const double4* nbr_v, unsigned int* queue, double* slot_acc, Slot<R>* slot_scr, int slot_stride,
          double* e3, double* sig3, unsigned long long* fxacc)
{
    extern __shared__ __align__(16) unsigned char smem[];
    EntryTile<R>* tiles = reinterpret_cast<EntryTile<R>*>(smem);
    __shared__ int s_root;
    __shared__ double wsum[kThreadsAtm / 32][13];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    constexpr int kWarps = kThreadsAtm / 32;
    double* acc = slot_acc + (size_t)blockIdx.x * slot_stride * kAcc;
    Slot<R>* scr = slot_scr + (size_t)blockIdx.x * slot_stride;
    EntryTile<R>& tl = tiles[wid];
    const R s9 = R(d.s9);
    const R alp = R(d.alp + 2.0);        // ATM exponent alp + 2 (rational.f90:563)
    const R alp3 = alp / R(3);
    const R cut2 = R(c.cut3 * c.cut3);
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
        const C6Entry<R>* msys = mat + mat_off[sys];
        const long long mrow_i = (long long)(i - a0) * nsys_n;
        const int orig_i = b.local[i];
        const int si = b.sp[i];
        // per-lane sums of this root: energy, dE/dCN, jk virial, accepted triples
        double e_root = 0.0, dei = 0.0;
        double sxx = 0, syy = 0, szz = 0, sxy = 0, sxz = 0, syz = 0;
        int ntrip = 0;
        if (m > 1) {
            // entry records of this root (all threads)
            for (int k = tid; k < m; k += kThreadsAtm) {
                const int j = nbr_j[base + k];
                double4 v = nbr_v[base + k];
                const bool ventry = v.w > 0.0;   // not an empty entry
                if (!ventry) v.w = 1.0;
                Slot<R> r;
                const int sj = b.sp[j];
                const C6Entry<R> e = msys[mrow_i + (j - a0)];
                const double r0 = __ldg(sp.atm_r0 + si * b.nid + sj);
                if constexpr (sizeof(R) == 8) {
                    r.v = make_double4(v.x, v.y, v.z, v.w);
                    r.l = make_double4(0.0, 0.0, 0.0, 1.0 / v.w);
                    r.c = make_double4(e.sc6, e.qrc, e.qcr, alp3 * (log(r0) - 0.5 * log(v.w)));
                    r.s = make_double4(rsqrt(v.w), 1.0, 0.0, 1.0);
                } else {
                    const float hx = __double2float_rn(v.x), hy = __double2float_rn(v.y), hz = __double2float_rn(v.z);
                    r.v = make_float4(hx, hy, hz, __double2float_rn(v.w));
                    r.l = make_float4(__double2float_rn(v.x - (double)hx), __double2float_rn(v.y - (double)hy),
                                      __double2float_rn(v.z - (double)hz), __double2float_rn(1.0 / v.w));
                    r.c = make_float4(e.sc6, e.qrc, e.qcr,
                                      __double2float_rn(double(alp3) * (log2(r0) - 0.5 * log2(v.w))));
                    r.s = make_float4(__double2float_rn(rsqrt(v.w)), 1.f, 0.f, 1.f);
                }
                if (SMOOTH) {
                    R sw, dsw;
                    const R rr = R(sqrt(v.w));
                    smooth<R>(rr, cutoff, width, sw, dsw);
                    r.s.y = sw;
                    r.s.z = dsw / rr;
                }
                r.meta = make_int4(j, 0, sj, b.local[j]);
                if (!ventry) { r.c.x = R(0); r.s.w = R(0); }
                scr[k] = r;
                if (GRAD)
                    for (int v2 = 0; v2 < kAcc; v2++) acc[k * kAcc + v2] = 0.0;
            }
            __syncthreads();
            const int T = (m + 31) >> 5;
            const int tp = T + (T & 1);
            // rounds 0 .. tp - 2: disjoint pairs of different tiles; round tp - 1: the tiles with themselves
            for (int round = 0; round < tp; round++) {
                const bool diag = round == tp - 1;
                const int npairs = diag ? T : tp / 2;
                for (int pk = wid; pk < npairs; pk += kWarps) {
                    int ta, tb;
                    if (diag) { ta = pk; tb = pk; }
                    else {
                        int x, y;
                        rr_pair(round, pk, tp, x, y);
                        if (x >= T || y >= T) continue;   // the pad tile of an odd tile count
                        ta = x > y ? x : y; tb = x > y ? y : x;
                    }
                    // row entry of this lane (registers), column entries (warp tile)
                    const int ea = 32 * ta + lane, eb = 32 * tb + lane;
                    const bool arow = ea < m;
                    Slot<R> A;
                    if (arow) A = scr[ea];
                    else {
                        A = scr[0];
                        A.c.x = R(0); A.s.w = R(0);
                    }
                    __syncwarp();
                    if (eb < m) {
                        const Slot<R> Bown = diag ? A : scr[eb];
                        tl.v[lane] = Bown.v; tl.l[lane] = Bown.l; tl.c[lane] = Bown.c; tl.s[lane] = Bown.s;
                        tl.meta[lane] = Bown.meta;
                    } else {
                        tl.v[lane] = A.v; tl.l[lane] = A.l; tl.c[lane] = A.c; tl.s[lane] = A.s;
                        tl.s[lane].w = R(0);
                        tl.c[lane].x = R(0);
                        tl.meta[lane] = A.meta;
                    }
                    __syncwarp();
                    const C6Entry<R>* row_a = msys + (long long)(A.meta.x - a0) * nsys_n;
                    const int t0 = diag ? 1 : 0, t1 = diag ? 16 : 31;
                    R kS = R(0), kGx = R(0), kGy = R(0), kGz = R(0), kD = R(0);
                    R rS = R(0), rGx = R(0), rGy = R(0), rGz = R(0), rD = R(0), rde = R(0);
                    R te = R(0), txx = R(0), tyy = R(0), tzz = R(0), txy = R(0), txz = R(0), tyz = R(0);
                    for (int st = t0; st <= t1; st++) {
                        const int mm = (lane + st) & 31;
                        const typename Vec4<R>::type Bv = tl.v[mm], Bl = tl.l[mm], Bc = tl.c[mm], Bs = tl.s[mm];
                        const int4 Bm = tl.meta[mm];
                        // C6 of the entry atoms (row a, column b): qrc = dC6/dCN_a / C6, qcr = dC6/dCN_b / C6
                        const C6Entry<R> ejk = row_a[Bm.x - a0];
                        // j-k vector: (x_k + T_k - x_i) - (x_j + T_j - x_i)
                        R vx, vy, vz;
                        if constexpr (sizeof(R) == 8) {
                            vx = Bv.x - A.v.x; vy = Bv.y - A.v.y; vz = Bv.z - A.v.z;
                        } else {
                            vx = (Bv.x - A.v.x) + (Bl.x - A.l.x);
                            vy = (Bv.y - A.v.y) + (Bl.y - A.l.y);
                            vz = (Bv.z - A.v.z) + (Bl.z - A.l.z);
                        }
                        const R rc0 = vx * vx + vy * vy + vz * vz;   // r_jk^2
                        bool valid = A.s.w != R(0) && Bs.w != R(0) && (!diag || st < 16 || lane < 16) &&
                                     !(rc0 > cut2 || rc0 < R(DBL_EPSILON));
                        // a step without any candidate inside the cutoff only moves the column sums
                        // (not for non-periodic systems in the FP32 form, where the test costs more
                        // than it saves)
                        if ((sizeof(R) == 4 && !PER) || __any_sync(0xffffffffu, valid)) {
                        if (part.nparts > 1) {
                            // owner of the triple: the pair of its two largest input indices
                            int o1 = orig_i, o2 = A.meta.w, o3 = Bm.w, tq;
                            if (o2 > o1) { tq = o1; o1 = o2; o2 = tq; }
                            if (o3 > o2) { tq = o2; o2 = o3; o3 = tq; }
                            if (o2 > o1) { tq = o1; o1 = o2; o2 = tq; }
                            valid = valid && owns_pair_atm(part, o1, o2);
                        }
                        const int jat = A.meta.x, kat = Bm.x;
                        // the reference's loop visits two images of one atom in both orders
                        ntrip += valid ? (jat == kat ? 2 : 1) : 0;
                        // triple_scale (atm.f90:954-980) of the atoms, twice for two images of one atom
                        R triple = R(1);
                        if (PER) {
                            if (jat == kat) triple = (i == jat) ? R(2.0 / 6.0) : R(1);
                            else triple = (i == jat || i == kat) ? R(0.5) : R(1);
                        }
                        const R rc = valid ? rc0 : R(1);
                        const R ra = A.v.w, rb = Bv.w;               // r_ij^2, r_ik^2
                        const R rsc = rsqrt_r<R>(rc);
                        const R irc = rsc * rsc;
                        const R ir1 = A.s.x * Bs.x * rsc;            // 1 / (r_ij r_ik r_jk)
                        const R ir2 = ir1 * ir1;
                        const R ir3 = ir2 * ir1;
                        const R ir5 = ir3 * ir2;
                        // (r0/r1)^alp3, r0 = r0ij r0ik r0jk, r1 = r_ij r_ik r_jk (atm.f90:744-749)
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
                        const R dE = (SMOOTH ? dE0 * sw : dE0) * triple;
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
                            if (PER) { sij *= triple; sik *= triple; sjk *= triple; }
                            const R gx = sjk * vx, gy = sjk * vy, gz = sjk * vz;
                            // dE/dCN: root share here, entry shares through the entry sums
                            const R hdE = R(0.5) * dE;
                            rde -= hdE * (A.c.y + Bc.y);
                            rS += sij; rGx -= gx; rGy -= gy; rGz -= gz;
                            rD -= hdE * (A.c.z + ejk.qrc);
                            kS += sik; kGx += gx; kGy += gy; kGz += gz;
                            kD -= hdE * (Bc.z + ejk.qcr);
                            txx += gx * vx; tyy += gy * vy; tzz += gz * vz;
                            txy += gx * vy; txz += gx * vz; tyz += gy * vz;
                        }
                        }
                        if (GRAD) {
                            // the column's sums move one lane down, with the column
                            const int src = (lane + 1) & 31;
                            kS = __shfl_sync(0xffffffffu, kS, src);
                            kGx = __shfl_sync(0xffffffffu, kGx, src);
                            kGy = __shfl_sync(0xffffffffu, kGy, src);
                            kGz = __shfl_sync(0xffffffffu, kGz, src);
                            kD = __shfl_sync(0xffffffffu, kD, src);
                        }
                    }
                    e_root += double(te);
                    if (GRAD) {
                        dei += double(rde);
                        sxx += double(txx); syy += double(tyy); szz += double(tzz);
                        sxy += double(txy); sxz += double(txz); syz += double(tyz);
                        // entry sums: the row's in this lane, the column (lane + t1 + 1) mod 32's too
                        if (arow) {
                            double* ar = acc + (size_t)ea * kAcc;
                            ar[0] += double(rS); ar[1] += double(rGx); ar[2] += double(rGy); ar[3] += double(rGz);
                            ar[4] += double(rD);
                        }
                        const int ef = 32 * tb + ((lane + t1 + 1) & 31);
                        if (ef < m) {
                            double* ak = acc + (size_t)ef * kAcc;
                            ak[0] += double(kS); ak[1] += double(kGx); ak[2] += double(kGy); ak[3] += double(kGz);
                            ak[4] += double(kD);
                        }
                    }
                    __syncwarp();
                }
                __syncthreads();
            }
        }
        // per-entry results: the root share stays in registers, the force and
        // dE/dCN share of the entry's atom go to its fixed-point accumulators
        double gix = 0, giy = 0, giz = 0;
        if (GRAD && m > 1) {
            for (int k = tid; k < m; k += kThreadsAtm) {
                const double S = acc[k * kAcc + 0];
                const double Gx = acc[k * kAcc + 1], Gy = acc[k * kAcc + 2], Gz = acc[k * kAcc + 3];
                const double Dx = acc[k * kAcc + 4];
                const double4 v = nbr_v[base + k];
                gix -= S * v.x; giy -= S * v.y; giz -= S * v.z;
                sxx += S * v.x * v.x; syy += S * v.y * v.y; szz += S * v.z * v.z;
                sxy += S * v.x * v.y; sxz += S * v.x * v.z; syz += S * v.y * v.z;
                unsigned long long* fx = fxacc + (size_t)8 * nbr_j[base + k];
                fixed_add(fx + 0, S * v.x + Gx);
                fixed_add(fx + 2, S * v.y + Gy);
                fixed_add(fx + 4, S * v.z + Gz);
                fixed_add(fx + 6, Dx);
            }
        }
        // block reduction of the root's sums in a fixed order
        double r[12] = {e_root, gix, giy, giz, dei, sxx, syy, szz, sxy, sxz, syz, double(ntrip)};
        for (int v = 0; v < 12; v++)
            for (int o = 16; o > 0; o >>= 1) r[v] += __shfl_xor_sync(0xffffffffu, r[v], o);
        if (lane == 0)
            for (int v = 0; v < 12; v++) wsum[wid][v] = r[v];
        __syncthreads();
        if (tid == 0) {
            double t[12] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
            for (int wq = 0; wq < kWarps; wq++)
                for (int v = 0; v < 12; v++) t[v] += wsum[wq][v];
            e3[i] = t[0];
            if (w.counts) atomicAdd(w.counts + 1, (unsigned long long)t[11]);
            if (GRAD) {
                unsigned long long* fx = fxacc + (size_t)8 * i;
                fixed_add(fx + 0, t[1]);
                fixed_add(fx + 2, t[2]);
                fixed_add(fx + 4, t[3]);
                fixed_add(fx + 6, t[4]);
                for (int v = 0; v < 6; v++) sig3[kSigma * i + v] = t[5 + v];
            }
        }
    }
}

// Adds the fixed-point three-body sums of every atom (gradient, dE/dCN) to
// the FP64 gradient and dE/dCN.
__global__ void k_atm_fixed(int natoms, const unsigned long long* fxacc, const int* guard, Work w)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= natoms || *guard) return;
    const unsigned long long* f = fxacc + (size_t)8 * x;
    w.grad[3 * x + 0] += fixed_value(f + 0);
    w.grad[3 * x + 1] += fixed_value(f + 2);
    w.grad[3 * x + 2] += fixed_value(f + 4);
    w.dEdcn[x] += fixed_value(f + 6);
}

}  // namespace

void launch_atm_fixed(int natoms, const unsigned long long* fxacc, const int* guard, const Work& w,
                      cudaStream_t stream)
{
    if (natoms <= 0) return;
    k_atm_fixed<<<(natoms + 255) / 256, 256, 0, stream>>>(natoms, fxacc, guard, w);
}

size_t atm_c6_entry_bytes(bool mixed) { return mixed ? sizeof(C6Entry<float>) : sizeof(C6Entry<double>); }

void launch_c6_matrix(const Batch& b, const Species& s, const Work& w, const void* U, double alp3,
                      const long long* d_mat_off, void* mat, long long total, bool mixed, cudaStream_t stream)
{
    if (total <= 0 || b.natoms <= 0) return;
    const unsigned blocks = (unsigned)((b.natoms + 7) / 8);
    if (mixed)
        k_c6_matrix<float><<<blocks, 256, 0, stream>>>(b, s, w, (const float*)U, alp3, d_mat_off, (C6Entry<float>*)mat);
    else
        k_c6_matrix<double><<<blocks, 256, 0, stream>>>(b, s, w, (const double*)U, alp3, d_mat_off,
                                                        (C6Entry<double>*)mat);
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

void launch_nbr_fill(const Batch& b, const Config& c, const uint8_t* sys_skip, const long long* off, const int* cnt,
                     int* nbr_j, int* nbr_gend, double4* nbr_v, const int* guard, cudaStream_t stream)
{
    if (b.natoms <= 0) return;
    k_nbr_fill<<<(b.natoms + 7) / 8, 256, 0, stream>>>(b, c, sys_skip, off, cnt, nbr_j, nbr_gend, nbr_v, guard);
}

template <class R>
size_t triple_smem()
{
    return sizeof(EntryTile<R>) * (kThreadsAtm / 32);
}

template <class R, bool GRAD, bool PER, bool SMOOTH>
int triple_occupancy_of()
{
    static bool configured = false;
    if (!configured) {
        cudaFuncSetAttribute(k_triples<R, GRAD, PER, SMOOTH>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)triple_smem<R>());
        configured = true;
    }
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_triples<R, GRAD, PER, SMOOTH>, kThreadsAtm, triple_smem<R>());
    return n > 0 ? n : 1;
}

template <class R, bool GRAD>
int triple_occupancy()
{
    // every variant is configured; the occupancy is the smallest of them
    return std::min(std::min(triple_occupancy_of<R, GRAD, false, false>(), triple_occupancy_of<R, GRAD, true, false>()),
                    std::min(triple_occupancy_of<R, GRAD, false, true>(), triple_occupancy_of<R, GRAD, true, true>()));
}

int atm_blocks_per_sm(bool mixed, bool grad)
{
    if (mixed) return grad ? triple_occupancy<float, true>() : triple_occupancy<float, false>();
    return grad ? triple_occupancy<double, true>() : triple_occupancy<double, false>();
}

size_t atm_slot_bytes(bool mixed) { return mixed ? sizeof(Slot<float>) : sizeof(Slot<double>); }

template <class R, bool GRAD, bool PER, bool SMOOTH>
void launch_triples_t(const Batch& b, const Species& s, const Damp& d, const Config& c, const Partition& p,
                      const Work& w, const void* mat, const long long* mat_off, const long long* off, const int* cnt,
                      const int* nbr_j, const int* nbr_gend, const double4* nbr_v, unsigned int* queue,
                      double* slot_acc, void* slot_scr, int slot_stride, int blocks, double* e3, double* sig3,
                      unsigned long long* fxacc, cudaStream_t stream)
{
    triple_occupancy_of<R, GRAD, PER, SMOOTH>();
    k_triples<R, GRAD, PER, SMOOTH><<<blocks, kThreadsAtm, triple_smem<R>(), stream>>>(
        b, s, d, c, p, w, (const C6Entry<R>*)mat, mat_off, off, cnt, nbr_j, nbr_gend, nbr_v, queue, slot_acc,
        (Slot<R>*)slot_scr, slot_stride, e3, sig3, fxacc);
}

template <class R, bool GRAD>
void launch_triples_g(const Batch& b, const Species& s, const Damp& d, const Config& c, const Partition& p,
                      const Work& w, const void* mat, const long long* mat_off, const long long* off, const int* cnt,
                      const int* nbr_j, const int* nbr_gend, const double4* nbr_v, unsigned int* queue,
                      double* slot_acc, void* slot_scr, int slot_stride, int blocks, bool periodic, double* e3,
                      double* sig3, unsigned long long* fxacc, cudaStream_t stream)
{
    const bool smooth_on = c.width3 > 0.0 && c.width3 < c.cut3;
#define D3_TRIPLES(P, S)                                                                                     \
    launch_triples_t<R, GRAD, P, S>(b, s, d, c, p, w, mat, mat_off, off, cnt, nbr_j, nbr_gend, nbr_v, queue,  \
                                    slot_acc, slot_scr, slot_stride, blocks, e3, sig3, fxacc, stream)
    if (periodic) { if (smooth_on) D3_TRIPLES(true, true); else D3_TRIPLES(true, false); }
    else { if (smooth_on) D3_TRIPLES(false, true); else D3_TRIPLES(false, false); }
#undef D3_TRIPLES
}

void launch_triples(const Batch& b, const Species& s, const Damp& d, const Config& c, const Partition& p,
                    const Work& w, const void* mat, const long long* mat_off, const long long* off, const int* cnt,
                    const int* nbr_j, const int* nbr_gend, const double4* nbr_v, unsigned int* queue,
                    double* slot_acc, void* slot_scr, int slot_stride, int blocks, bool periodic, double* e3,
                    double* sig3, unsigned long long* fxacc, cudaStream_t stream)
{
    if (b.natoms <= 0) return;
    if (c.mixed) {
        if (c.grad) launch_triples_g<float, true>(b, s, d, c, p, w, mat, mat_off, off, cnt, nbr_j, nbr_gend, nbr_v, queue, slot_acc, slot_scr, slot_stride, blocks, periodic, e3, sig3, fxacc, stream);
        else launch_triples_g<float, false>(b, s, d, c, p, w, mat, mat_off, off, cnt, nbr_j, nbr_gend, nbr_v, queue, slot_acc, slot_scr, slot_stride, blocks, periodic, e3, sig3, fxacc, stream);
    } else {
        if (c.grad) launch_triples_g<double, true>(b, s, d, c, p, w, mat, mat_off, off, cnt, nbr_j, nbr_gend, nbr_v, queue, slot_acc, slot_scr, slot_stride, blocks, periodic, e3, sig3, fxacc, stream);
        else launch_triples_g<double, false>(b, s, d, c, p, w, mat, mat_off, off, cnt, nbr_j, nbr_gend, nbr_v, queue, slot_acc, slot_scr, slot_stride, blocks, periodic, e3, sig3, fxacc, stream);
    }
}

}  // namespace d3
