// Spatially ordered, tile-culled pair sweeps: coordination number, two-body
// dispersion and CN chain rule.
//
// Atoms of every system are put in Morton order (cub radix sort of quantised
// positions), and each run of 32 consecutive atoms of a system forms a tile
// with a bounding sphere.  A warp owns one atom i: it stages y(T) = x_i - T for
// a chunk of lattice translations in shared memory, tests all 32 atoms of a
// tile against 32 translations at once with the tile's bounding sphere (one
// ballot per 32 translations), and evaluates the pair terms only for the
// translations that can reach the tile, one j per lane.  The work per pair
// term is the same as in the unsorted kernels; the candidate tests that the
// cutoff rejects anyway are skipped in blocks of 32.
//
// C6 interpolation uses per-warp species vectors: for the warp's atom i and
// every species s, u_s = sum_r gw_i[r] C6ref(r, ., si, s) and the same with
// dgw_i, so C6_ij and its two CN derivatives cost 3 short dot products per j
// (get_atomic_c6, model.f90:432-461).
#include <cub/cub.cuh>

#include <algorithm>
#include <cfloat>
#include <cstdint>

#include "d3_device.cuh"

namespace d3 {

namespace {

constexpr int kChunk = 128;            // translations staged per pass (4 ballot words)
constexpr int kOrderThreads = 128;      // threads of the per-system shape blocks
constexpr int kMaxColumns = 64;         // slabs per system and columns per slab at most (12-bit groups)
constexpr double kKcn = 16.0;          // ncoord.f90:31

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    return v;
}

__device__ __forceinline__ bool owns_pair(const Partition& p, int i, int j)
{
    // partition.f90:127-147 on zero-based system-local input indices
    if (p.nparts <= 1) return true;
    long long hi = i > j ? i : j, lo = i > j ? j : i;
    return (hi * (hi + 1) / 2 + lo) % p.nparts == p.part;
}

struct Sh64 { double x, y, z; };
struct Sh32 { float4 hi, lo; };
template <class R> struct ShOf;
template <> struct ShOf<double> { using type = Sh64; };
template <> struct ShOf<float> { using type = Sh32; };

__device__ __forceinline__ Sh32 split3(double x, double y, double z)
{
    Sh32 s;
    s.hi = make_float4(__double2float_rn(x), __double2float_rn(y), __double2float_rn(z), 0.f);
    s.lo = make_float4(__double2float_rn(x - (double)s.hi.x), __double2float_rn(y - (double)s.hi.y),
                       __double2float_rn(z - (double)s.hi.z), 0.f);
    return s;
}

__device__ __forceinline__ void pos_of(const Sh64& s, double& x, double& y, double& z) { x = s.x; y = s.y; z = s.z; }
__device__ __forceinline__ void pos_of(const Sh32& s, double& x, double& y, double& z)
{
    x = (double)s.hi.x + (double)s.lo.x;
    y = (double)s.hi.y + (double)s.lo.y;
    z = (double)s.hi.z + (double)s.lo.z;
}

__device__ __forceinline__ void disp(const Sh64& s, double xj, double yj, double zj, float4, float4,
                                     double& vx, double& vy, double& vz)
{
    vx = s.x - xj; vy = s.y - yj; vz = s.z - zj;
}

__device__ __forceinline__ void disp(const Sh32& s, double, double, double, float4 hj, float4 lj,
                                     float& vx, float& vy, float& vz)
{
    vx = (s.hi.x - hj.x) + (s.lo.x - lj.x);
    vy = (s.hi.y - hj.y) + (s.lo.y - lj.y);
    vz = (s.hi.z - hj.z) + (s.lo.z - lj.z);
}

template <class R>
__device__ __forceinline__ void stage(typename ShOf<R>::type* buf, const double* img, int t0, int nt, double xi,
                                      double yi, double zi, int lane)
{
    for (int k = lane; k < nt; k += 32) {
        const double tx = __ldg(img + 3 * (t0 + k)), ty = __ldg(img + 3 * (t0 + k) + 1), tz = __ldg(img + 3 * (t0 + k) + 2);
        if constexpr (sizeof(R) == 8) buf[k] = Sh64{xi - tx, yi - ty, zi - tz};
        else buf[k] = split3(xi - tx, yi - ty, zi - tz);
    }
    __syncwarp();
}

// Ballot of the staged translations [32 w, 32 w + 32) that can reach a tile.
template <class R>
__device__ __forceinline__ unsigned reach(const typename ShOf<R>::type* buf, int nt, int w, int lane, double4 tb,
                                          double cutoff)
{
    const int k = 32 * w + lane;
    bool ok = false;
    if (k < nt) {
        double yx, yy, yz;
        pos_of(buf[k], yx, yy, yz);
        const double dx = yx - tb.x, dy = yy - tb.y, dz = yz - tb.z;
        const double lim = cutoff + tb.w + 1.0e-6 * cutoff + 1.0e-6;
        ok = dx * dx + dy * dy + dz * dz <= lim * lim;
    }
    return __ballot_sync(0xffffffffu, ok);
}

// Reciprocal and reciprocal square root of the pair arithmetic: IEEE in the
// FP64 form, the hardware approximations (a few ulp) in the FP32 part of the
// mixed form.
template <class R> __device__ __forceinline__ R r_rcp(R x) { if constexpr (sizeof(R) == 8) return R(1) / x; else return __fdividef(1.0f, x); }
template <class R> __device__ __forceinline__ R r_rsqrt(R x) { if constexpr (sizeof(R) == 8) return R(1) / sqrt(x); else return rsqrtf(x); }
template <class R> __device__ __forceinline__ R r_sqrt(R x) { if constexpr (sizeof(R) == 8) return sqrt(x); else return sqrtf(x); }
template <class R> __device__ __forceinline__ R r_exp(R x) { if constexpr (sizeof(R) == 8) return exp(x); else return expf(x); }
template <class R> __device__ __forceinline__ R r_pow(R x, R a) { if constexpr (sizeof(R) == 8) return pow(x, a); else return powf(x, a); }

template <class R>
__device__ __forceinline__ void smooth(R r, R cutoff, R width, R& sw, R& dswdr)
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

// Counting function 1 / (1 + exp(-kcn (rc / r - 1))) (ncoord.f90:124-131);
// optionally returns 1 / r.
template <class R>
__device__ __forceinline__ R r_cn_count(R rc, R r2, R* inv_r = nullptr)
{
    if constexpr (sizeof(R) == 8) {
        const R r1 = sqrt(r2);
        if (inv_r) *inv_r = R(1) / r1;
        return R(1) / (R(1) + exp(-R(kKcn) * (rc / r1 - R(1))));
    } else {
        const R ir = rsqrtf(r2);
        if (inv_r) *inv_r = ir;
        return __fdividef(1.0f, 1.0f + expf(-R(kKcn) * (rc * ir - R(1))));
    }
}

struct Range {
    int j0, j1, t0, t1, tile0;
};

__device__ __forceinline__ Range range_of(const Batch& b, int i, int kind)
{
    const int sys = b.sys_of_atom[i];
    Range r;
    r.j0 = b.atom_off[sys];
    r.j1 = b.atom_off[sys + 1];
    r.t0 = b.img_off[kind * (b.nsys + 1) + sys];
    r.t1 = b.img_off[kind * (b.nsys + 1) + sys + 1];
    r.tile0 = b.tile_off[sys];
    return r;
}

// ----------------------------------------------------- coordination number --

template <int W, class R>
__global__ void __launch_bounds__(32 * W, 16 / W) k_cn_tiled(Batch b, Species s, Config c, Partition p, Work w)
{
    using Sh = typename ShOf<R>::type;
    __shared__ Sh sbuf[W][kChunk];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int i = blockIdx.x * W + wib;
    if (i >= b.natoms) return;
    const Range rg = range_of(b, i, kImgCN);
    const double xi = b.x[i], yi = b.y[i], zi = b.z[i];
    const double rci = s.rcov[b.sp[i]];
    const int li = b.local[i];
    const R cut2 = R(c.cut_cn * c.cut_cn);
    double acc = 0.0;
    R tacc = R(0);
    unsigned long long nterm = 0;
    for (int tc = rg.t0; tc < rg.t1; tc += kChunk) {
        const int nt = min(kChunk, rg.t1 - tc);
        stage<R>(sbuf[wib], b.img, tc, nt, xi, yi, zi, lane);
        const int nw = (nt + 31) / 32;
        for (int jb = rg.j0, tile = rg.tile0; jb < rg.j1; jb += kTile, tile++) {
            const double4 tb = b.tiles[tile];
            unsigned mk[4] = {0u, 0u, 0u, 0u};
            unsigned any = 0u;
#pragma unroll
            for (int q = 0; q < 4; q++)
                if (q < nw) { mk[q] = reach<R>(sbuf[wib], nt, q, lane, tb, c.cut_cn); any |= mk[q]; }
            if (!any) continue;
            const int j = jb + lane;
            const bool valid = j < rg.j1 && (!c.cn_partitioned || owns_pair(p, li, b.local[j < rg.j1 ? j : rg.j0]));
            const int jj = j < rg.j1 ? j : rg.j0;
            const double xj = b.x[jj], yj = b.y[jj], zj = b.z[jj];
            float4 hj = make_float4(0, 0, 0, 0), lj = hj;
            if constexpr (sizeof(R) == 4) { hj = b.xhi[jj]; lj = b.xlo[jj]; }
            const R rc = R(rci + s.rcov[b.sp[jj]]);
            if constexpr (sizeof(R) == 4) tacc = R(0);
#pragma unroll
            for (int q = 0; q < 4; q++) {
                unsigned m = mk[q];
                while (m) {
                    const int k = 32 * q + __ffs(m) - 1;
                    m &= m - 1;
                    R vx, vy, vz;
                    disp(sbuf[wib][k], xj, yj, zj, hj, lj, vx, vy, vz);
                    const R r2 = vx * vx + vy * vy + vz * vz;
                    if (!valid || r2 > cut2 || r2 < R(1.0e-12)) continue;
                    tacc += r_cn_count<R>(rc, r2);
                    nterm += (jj <= i);
                }
            }
            if constexpr (sizeof(R) == 4) acc += double(tacc);
        }
        __syncwarp();
    }
    if constexpr (sizeof(R) == 8) acc = tacc;
    acc = warp_sum(acc);
    if (lane == 0) w.cn[i] = acc;
    if (w.counts) {
        for (int off = 16; off > 0; off >>= 1) nterm += __shfl_xor_sync(0xffffffffu, nterm, off);
        if (lane == 0) atomicAdd(w.counts + 2, nterm);
    }
}

// ---------------------------------------------------------------- two-body --

template <int W, class R, int DAMP>
__global__ void __launch_bounds__(32 * W, 16 / W) k_two_body_tiled(Batch b, Species s, Damp d, Config c, Partition p,
                                                             Work w)
{
    using Sh = typename ShOf<R>::type;
    __shared__ Sh sbuf[W][kChunk];
    __shared__ R su[W][kMaxSpeciesFast][kMaxRef];
    __shared__ R sdu[W][kMaxSpeciesFast][kMaxRef];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int i = blockIdx.x * W + wib;
    if (i >= b.natoms) return;
    const Range rg = range_of(b, i, kImgDisp2);
    const double xi = b.x[i], yi = b.y[i], zi = b.z[i];
    const int si = b.sp[i], nid = b.nid;
    const int nri = s.nref[si];
    const int li = b.local[i];
    const bool gi = b.ghost && b.ghost[i];
    // species vectors of atom i: u[sj][jr] = sum_ir gw_i[ir] c6(ir, jr, si, sj)
    for (int idx = lane; idx < nid * kMaxRef; idx += 32) {
        const int sj = idx / kMaxRef, jr = idx % kMaxRef;
        R u = R(0), du = R(0);
        if (!gi && jr < s.nref[sj]) {
            const int base = (si * nid + sj) * kMaxRef * kMaxRef;
            for (int ir = 0; ir < nri; ir++) {
                R ref, g, dg;
                if constexpr (sizeof(R) == 8) {
                    ref = __ldg(s.c6ref + base + ir * kMaxRef + jr);
                    g = w.gw[i * kMaxRef + ir]; dg = w.dgw[i * kMaxRef + ir];
                } else {
                    ref = __ldg(s.c6ref_f + base + ir * kMaxRef + jr);
                    g = w.gwf[i * kMaxRef + ir]; dg = w.dgwf[i * kMaxRef + ir];
                }
                u += g * ref;
                du += dg * ref;
            }
        }
        su[wib][sj][jr] = u;
        sdu[wib][sj][jr] = du;
    }
    __syncwarp();
    const R cutoff = R(c.cut2), cut2 = R(c.cut2 * c.cut2), width = R(c.width2);
    const bool smooth_on = c.width2 > 0.0 && c.width2 < c.cut2;
    const R s6 = R(d.s6), s8 = R(d.s8);
    const R alp6 = R(d.alp), alp8 = R(d.alp + 2.0);
    double e = 0, de = 0, gx = 0, gy = 0, gz = 0;
    double sxx = 0, syy = 0, szz = 0, sxy = 0, sxz = 0, syz = 0;
    double pg0 = 0, pg1 = 0, pg2 = 0, pg3 = 0;
    R te = R(0), tde = R(0), tgx = R(0), tgy = R(0), tgz = R(0);
    R txx = R(0), tyy = R(0), tzz = R(0), txy = R(0), txz = R(0), tyz = R(0);
    R tp0 = R(0), tp1 = R(0), tp2 = R(0), tp3 = R(0);
    unsigned long long nterm = 0;
    for (int tc = rg.t0; tc < rg.t1; tc += kChunk) {
        const int nt = min(kChunk, rg.t1 - tc);
        stage<R>(sbuf[wib], b.img, tc, nt, xi, yi, zi, lane);
        const int nw = (nt + 31) / 32;
        for (int jb = rg.j0, tile = rg.tile0; jb < rg.j1; jb += kTile, tile++) {
            const double4 tb = b.tiles[tile];
            unsigned mk[4] = {0u, 0u, 0u, 0u};
            unsigned any = 0u;
#pragma unroll
            for (int q = 0; q < 4; q++)
                if (q < nw) { mk[q] = reach<R>(sbuf[wib], nt, q, lane, tb, c.cut2); any |= mk[q]; }
            if (!any) continue;
            const int j = jb + lane;
            const int jj = j < rg.j1 ? j : rg.j0;
            const bool valid = j < rg.j1 && owns_pair(p, li, b.local[jj]);
            const double xj = b.x[jj], yj = b.y[jj], zj = b.z[jj];
            float4 hj = make_float4(0, 0, 0, 0), lj = hj;
            if constexpr (sizeof(R) == 4) { hj = b.xhi[jj]; lj = b.xlo[jj]; }
            const int sj = b.sp[jj];
            R c6 = R(0), dc6i = R(0), dc6j = R(0);
            if (valid && !(b.ghost && b.ghost[jj])) {
                const int nrj = s.nref[sj];
                for (int jr = 0; jr < nrj; jr++) {
                    R g, dg;
                    if constexpr (sizeof(R) == 8) { g = w.gw[jj * kMaxRef + jr]; dg = w.dgw[jj * kMaxRef + jr]; }
                    else { g = w.gwf[jj * kMaxRef + jr]; dg = w.dgwf[jj * kMaxRef + jr]; }
                    const R u = su[wib][sj][jr], du = sdu[wib][sj][jr];
                    c6 += u * g;
                    dc6i += du * g;
                    dc6j += u * dg;
                }
            }
            const double* pr = s.pair + kPairSlots * (si * nid + sj);
            const R rrij = R(__ldg(pr + 0));
            const R q1 = R(__ldg(pr + 1)), q2 = R(__ldg(pr + 2)), q3 = R(__ldg(pr + 3)), q4 = R(__ldg(pr + 4));
            // mixed form: FP32 partial sums over the translations of this tile,
            // added to the FP64 accumulators once per tile
            if constexpr (sizeof(R) == 4) {
                te = tde = tgx = tgy = tgz = R(0);
                txx = tyy = tzz = txy = txz = tyz = R(0);
                tp0 = tp1 = tp2 = tp3 = R(0);
            }
#pragma unroll
            for (int q = 0; q < 4; q++) {
                unsigned m = mk[q];
                while (m) {
                    const int k = 32 * q + __ffs(m) - 1;
                    m &= m - 1;
                    R vx, vy, vz;
                    disp(sbuf[wib][k], xj, yj, zj, hj, lj, vx, vy, vz);
                    const R r2 = vx * vx + vy * vy + vz * vz;
                    if (!valid || r2 > cut2 || r2 < R(DBL_EPSILON)) continue;
                    nterm += (jj <= i);   // the reference's (i, j <= i, T) count
                    R sw = R(1), dswdr = R(0), r1 = R(0);
                    if (smooth_on) { r1 = r_sqrt<R>(r2); smooth<R>(r1, cutoff, width, sw, dswdr); }
                    R edisp0, gdisp0, e6, e8, dpa = R(0), dpb = R(0);
                    if constexpr (DAMP == kRational) {
                        // rational.f90:462-497: q1 = R0^6, q2 = R0^8, q3 = R0, q4 = sqrt(rrij)
                        const R r4 = r2 * r2;
                        const R a6 = r4 * r2 + q1, a8 = r4 * r4 + q2;
                        const R inv = r_rcp<R>(a6 * a8);
                        const R t6 = a8 * inv;
                        const R t8 = a6 * inv;
                        const R d6 = R(-6) * r4 * t6 * t6;
                        const R d8 = R(-8) * r4 * r2 * t8 * t8;
                        e6 = t6; e8 = rrij * t8;
                        edisp0 = s6 * t6 + s8 * rrij * t8;
                        gdisp0 = s6 * d6 + s8 * rrij * d8;
                        if (c.param_grad) {
                            const R dedr0 = s6 * R(-6) * (q1 / q3) * t6 * t6 + s8 * rrij * R(-8) * (q2 / q3) * t8 * t8;
                            dpa = dedr0 * q4;
                            dpb = dedr0;
                        }
                    } else {
                        // zero.f90:490-536: q1 = rs6 R0, q2 = rs8 R0
                        if (!smooth_on) r1 = r_sqrt<R>(r2);
                        const R r6 = r2 * r2 * r2;
                        const R r8 = r6 * r2;
                        const R t6 = r_pow<R>(q1 / r1, alp6);
                        const R t8 = r_pow<R>(q2 / r1, alp8);
                        const R f6 = R(1) / (R(1) + R(6) * t6);
                        const R f8 = R(1) / (R(1) + R(6) * t8);
                        const R d6 = R(-6) * f6 / r2 + R(6) * alp6 * t6 * (f6 * f6) / r2;
                        const R d8 = R(-8) * f8 / r2 + R(6) * alp8 * t8 * (f8 * f8) / r2;
                        e6 = f6 / r6; e8 = rrij * f8 / r8;
                        edisp0 = s6 * f6 / r6 + s8 * rrij * f8 / r8;
                        gdisp0 = s6 * d6 / r6 + s8 * rrij * d8 / r8;
                        if (c.param_grad) {
                            dpa = d.rs6 != 0.0 ? s6 / r6 * R(-6) * f6 * f6 * alp6 * t6 / R(d.rs6) : R(0);
                            dpb = d.rs8 != 0.0 ? s8 * rrij / r8 * R(-6) * f8 * f8 * alp8 * t8 / R(d.rs8) : R(0);
                        }
                    }
                    const R edisp = sw * edisp0;
                    te += -c6 * edisp * R(0.5);
                    tde -= dc6i * edisp;
                    if (c.param_grad) {
                        const R hc = R(-0.5) * c6 * sw;
                        tp0 += hc * e6; tp1 += hc * e8;
                        tp2 += hc * dpa; tp3 += hc * dpb;
                    }
                    if (!c.grad) continue;
                    R gdisp = sw * gdisp0;
                    if (smooth_on) gdisp += dswdr * edisp0 / r1;
                    const R f = -c6 * gdisp;
                    const R dgx = f * vx, dgy = f * vy, dgz = f * vz;
                    if (jj != i) { tgx += dgx; tgy += dgy; tgz += dgz; }
                    txx += dgx * vx; tyy += dgy * vy; tzz += dgz * vz;
                    txy += dgx * vy; txz += dgx * vz; tyz += dgy * vz;
                }
            }
            if constexpr (sizeof(R) == 4) {
                e += double(te);
                de += double(tde);
                if (c.param_grad) { pg0 += double(tp0); pg1 += double(tp1); pg2 += double(tp2); pg3 += double(tp3); }
                if (c.grad) {
                    gx += double(tgx); gy += double(tgy); gz += double(tgz);
                    sxx += double(txx); syy += double(tyy); szz += double(tzz);
                    sxy += double(txy); sxz += double(txz); syz += double(tyz);
                }
            }
        }
        __syncwarp();
    }
    if constexpr (sizeof(R) == 8) {
        // the FP64 form accumulates directly in the tile sums
        e = te; de = tde; pg0 = tp0; pg1 = tp1; pg2 = tp2; pg3 = tp3;
        gx = tgx; gy = tgy; gz = tgz;
        sxx = txx; syy = tyy; szz = tzz; sxy = txy; sxz = txz; syz = tyz;
    }
    sxx *= 0.5; syy *= 0.5; szz *= 0.5; sxy *= 0.5; sxz *= 0.5; syz *= 0.5;
    e = warp_sum(e);
    if (lane == 0) w.e_atom[i] = e;
    if (c.grad) {
        de = warp_sum(de); gx = warp_sum(gx); gy = warp_sum(gy); gz = warp_sum(gz);
        sxx = warp_sum(sxx); syy = warp_sum(syy); szz = warp_sum(szz);
        sxy = warp_sum(sxy); sxz = warp_sum(sxz); syz = warp_sum(syz);
        if (lane == 0) {
            w.dEdcn[i] = de;
            w.grad[3 * i + 0] = gx; w.grad[3 * i + 1] = gy; w.grad[3 * i + 2] = gz;
            double* sg = w.sig_atom + kSigma * i;
            sg[0] = sxx; sg[1] = syy; sg[2] = szz; sg[3] = sxy; sg[4] = sxz; sg[5] = syz;
        }
    }
    if (c.param_grad) {
        pg0 = warp_sum(pg0); pg1 = warp_sum(pg1); pg2 = warp_sum(pg2); pg3 = warp_sum(pg3);
        if (lane == 0) {
            double* pg = w.pg_atom + kParamGrad * i;
            pg[0] = pg0; pg[1] = pg1; pg[2] = pg2; pg[3] = pg3;
        }
    }
    if (w.counts) {
        for (int off = 16; off > 0; off >>= 1) nterm += __shfl_xor_sync(0xffffffffu, nterm, off);
        if (lane == 0) atomicAdd(w.counts + 0, nterm);
    }
}

// ------------------------------------------------------------- chain rule --

template <int W, class R>
__global__ void __launch_bounds__(32 * W, 16 / W) k_chain_tiled(Batch b, Species s, Config c, Partition p, Work w)
{
    using Sh = typename ShOf<R>::type;
    __shared__ Sh sbuf[W][kChunk];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int i = blockIdx.x * W + wib;
    if (i >= b.natoms) return;
    const Range rg = range_of(b, i, kImgCN);
    const double xi = b.x[i], yi = b.y[i], zi = b.z[i];
    const double rci = s.rcov[b.sp[i]];
    const double dei = w.dEdcn[i];
    const int li = b.local[i];
    const R cut2 = R(c.cut_cn * c.cut_cn);
    double gx = 0, gy = 0, gz = 0, sxx = 0, syy = 0, szz = 0, sxy = 0, sxz = 0, syz = 0;
    R tgx = R(0), tgy = R(0), tgz = R(0), txx = R(0), tyy = R(0), tzz = R(0);
    R txy = R(0), txz = R(0), tyz = R(0);
    for (int tc = rg.t0; tc < rg.t1; tc += kChunk) {
        const int nt = min(kChunk, rg.t1 - tc);
        stage<R>(sbuf[wib], b.img, tc, nt, xi, yi, zi, lane);
        const int nw = (nt + 31) / 32;
        for (int jb = rg.j0, tile = rg.tile0; jb < rg.j1; jb += kTile, tile++) {
            const double4 tb = b.tiles[tile];
            unsigned mk[4] = {0u, 0u, 0u, 0u};
            unsigned any = 0u;
#pragma unroll
            for (int q = 0; q < 4; q++)
                if (q < nw) { mk[q] = reach<R>(sbuf[wib], nt, q, lane, tb, c.cut_cn); any |= mk[q]; }
            if (!any) continue;
            const int j = jb + lane;
            const int jj = j < rg.j1 ? j : rg.j0;
            const bool valid = j < rg.j1 && (!c.cn_partitioned || owns_pair(p, li, b.local[jj]));
            const double xj = b.x[jj], yj = b.y[jj], zj = b.z[jj];
            float4 hj = make_float4(0, 0, 0, 0), lj = hj;
            if constexpr (sizeof(R) == 4) { hj = b.xhi[jj]; lj = b.xlo[jj]; }
            const R rc = R(rci + s.rcov[b.sp[jj]]);
            // 0.5 (dEdcn_i + dEdcn_j) is this atom's virial share of the pair
            const R dsum = R(dei + w.dEdcn[jj]);
            if constexpr (sizeof(R) == 4) {
                tgx = tgy = tgz = txx = tyy = tzz = txy = txz = tyz = R(0);
            }
#pragma unroll
            for (int q = 0; q < 4; q++) {
                unsigned m = mk[q];
                while (m) {
                    const int k = 32 * q + __ffs(m) - 1;
                    m &= m - 1;
                    R vx, vy, vz;
                    disp(sbuf[wib][k], xj, yj, zj, hj, lj, vx, vy, vz);
                    const R r2 = vx * vx + vy * vy + vz * vz;
                    if (!valid || r2 > cut2 || r2 < R(1.0e-12)) continue;
                    R f;
                    if constexpr (sizeof(R) == 8) {
                        // ncoord.f90:198-206
                        const R r1 = sqrt(r2);
                        const R cf = R(1) / (R(1) + exp(-R(kKcn) * (rc / r1 - R(1))));
                        const R dcf = -cf * (R(1) - cf) * R(kKcn) * rc / r2;
                        f = dcf / r1 * dsum;
                    } else {
                        R irr;
                        const R cf = r_cn_count<R>(rc, r2, &irr);
                        // dcf / r = -cf (1 - cf) kcn rc / r^3
                        f = -cf * (R(1) - cf) * R(kKcn) * rc * (irr * irr * irr) * dsum;
                    }
                    const R cx = f * vx, cy = f * vy, cz = f * vz;
                    if (jj != i) { tgx += cx; tgy += cy; tgz += cz; }
                    txx += cx * vx; tyy += cy * vy; tzz += cz * vz;
                    txy += cx * vy; txz += cx * vz; tyz += cy * vz;
                }
            }
            if constexpr (sizeof(R) == 4) {
                gx += double(tgx); gy += double(tgy); gz += double(tgz);
                sxx += double(txx); syy += double(tyy); szz += double(tzz);
                sxy += double(txy); sxz += double(txz); syz += double(tyz);
            }
        }
        __syncwarp();
    }
    if constexpr (sizeof(R) == 8) {
        gx = tgx; gy = tgy; gz = tgz;
        sxx = txx; syy = tyy; szz = tzz; sxy = txy; sxz = txz; syz = tyz;
    }
    sxx *= 0.5; syy *= 0.5; szz *= 0.5; sxy *= 0.5; sxz *= 0.5; syz *= 0.5;
    gx = warp_sum(gx); gy = warp_sum(gy); gz = warp_sum(gz);
    sxx = warp_sum(sxx); syy = warp_sum(syy); szz = warp_sum(szz);
    sxy = warp_sum(sxy); sxz = warp_sum(sxz); syz = warp_sum(syz);
    if (lane == 0) {
        w.grad[3 * i + 0] += gx; w.grad[3 * i + 1] += gy; w.grad[3 * i + 2] += gz;
        double* sg = w.sig_atom + kSigma * i;
        sg[0] += sxx; sg[1] += syy; sg[2] += szz; sg[3] += sxy; sg[4] += sxz; sg[5] += syz;
    }
}

// ------------------------------------------------------- ordering, tiles ----

__device__ __forceinline__ unsigned long long spread3(unsigned v)
{
    unsigned long long x = v & 0x3ffu;
    x = (x | (x << 16)) & 0x030000FFull;
    x = (x | (x << 8)) & 0x0300F00Full;
    x = (x | (x << 4)) & 0x030C30C3ull;
    x = (x | (x << 2)) & 0x09249249ull;
    return x;
}

// Sort key: system index above a 30-bit Morton code of the position
// quantised to cells of `cell` Bohr.
__global__ void k_morton(const double* __restrict__ pos, int n, const int* sys_of_atom, double inv_cell,
                         unsigned long long* keys, int* idx)
{
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= n) return;
    unsigned q[3];
    for (int c = 0; c < 3; c++) {
        double f = floor(pos[3 * a + c] * inv_cell) + 512.0;
        f = fmin(fmax(f, 0.0), 1023.0);
        q[c] = (unsigned)f;
    }
    const unsigned long long m = spread3(q[0]) | (spread3(q[1]) << 1) | (spread3(q[2]) << 2);
    keys[a] = ((unsigned long long)sys_of_atom[a] << 30) | m;
    idx[a] = a;
}

// Column order.  Every system is cut into nx slabs along x, each slab into
// ny columns along y, and each column is ordered along z; slab and column
// boundaries fall on multiples of kTile atoms, so every tile of 32
// consecutive atoms is a compact box inside one column (a Morton curve puts
// atoms from distant cells into one tile wherever the curve jumps).
//
// Each of three passes gives every atom its position inside its system in
// the order of a 64-bit word (group, coordinate key, local index): pass 0
// orders by x, pass 1 by (slab, y), pass 2 by (slab * ny + column, z), where
// slab and column follow from the previous pass's position.  The position is
// a count over the atoms of the system by a group of lanes (O(n^2) per
// system, no sort and no barrier), the order of three stable sorts.  The shape kernel writes the
// pass-0 words, each pass the words of the next, the last pass the sorted
// atom arrays.

// Order-preserving 32-bit key of a coordinate.
__device__ __forceinline__ unsigned coord_key(double v)
{
    const unsigned u = __float_as_uint(__double2float_rn(v));
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

// Largest s with floor(s n / k) <= t: the part (of k parts of n tiles) that
// holds tile t.
__device__ __forceinline__ int part_of(int t, int n, int k)
{
    return (int)(((long long)(t + 1) * k - 1) / n);
}

__device__ __forceinline__ unsigned long long order_word(unsigned long long group, double coord, int li)
{
    return (group << 52) | ((unsigned long long)coord_key(coord) << 20) | (unsigned long long)li;
}

// Slabs and columns of every system from its bounding box, boxes of about
// equal edge holding one tile each; one block of BLOCK threads per system,
// which also writes the pass-0 words of its atoms.
__device__ __forceinline__ int2 system_shape(const double lo[3], const double hi[3], int nt)
{
    int nx = 1, ny = 1;
    if (nt > 1) {
        const double lx = fmax(hi[0] - lo[0], 1.0), ly = fmax(hi[1] - lo[1], 1.0), lz = fmax(hi[2] - lo[2], 1.0);
        const double edge = cbrt(lx * ly * lz / nt);
        nx = (int)fmin(fmax(rint(lx / edge), 1.0), (double)kMaxColumns);
        nx = min(nx, nt);
        ny = (int)fmin(fmax(rint(ly / edge), 1.0), (double)kMaxColumns);
        ny = max(1, min(ny, nt / nx));
    }
    return make_int2(nx, ny);
}

// Group of the next pass's word for the atom at position r of its system
// after pass PASS (0: slab, 1: slab * ny + column).
template <int PASS>
__device__ __forceinline__ unsigned long long order_group(int r, int nt, int2 sh)
{
    const int t = r / kTile;
    const int slab = part_of(t, nt, sh.x);
    if (PASS == 0) return (unsigned long long)slab;
    const int s0 = (int)((long long)slab * nt / sh.x), s1 = (int)((long long)(slab + 1) * nt / sh.x);
    return (unsigned long long)(slab * sh.y + part_of(t - s0, s1 - s0, sh.y));
}

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK)
k_rank_shape(const double* __restrict__ pos, const int* atom_off, const int* tile_off, int2* shape,
             unsigned long long* word)
{
    pdl_wait();
    __shared__ double red[6][BLOCK / 32];
    const int sys = blockIdx.x;
    const int a0 = atom_off[sys], a1 = atom_off[sys + 1];
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int a = a0 + threadIdx.x; a < a1; a += blockDim.x) {
        for (int c = 0; c < 3; c++) {
            const double v = pos[3 * a + c];
            lo[c] = fmin(lo[c], v);
            hi[c] = fmax(hi[c], v);
        }
        word[a] = order_word(0, pos[3 * a], a - a0);
    }
    for (int c = 0; c < 3; c++)
        for (int o = 16; o > 0; o >>= 1) {
            lo[c] = fmin(lo[c], __shfl_xor_sync(0xffffffffu, lo[c], o));
            hi[c] = fmax(hi[c], __shfl_xor_sync(0xffffffffu, hi[c], o));
        }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0)
        for (int c = 0; c < 3; c++) { red[c][wid] = lo[c]; red[3 + c][wid] = hi[c]; }
    __syncthreads();
    if (threadIdx.x != 0) return;
    for (int w = 1; w < BLOCK / 32; w++)
        for (int c = 0; c < 3; c++) {
            lo[c] = fmin(lo[c], red[c][w]);
            hi[c] = fmax(hi[c], red[3 + c][w]);
        }
    shape[sys] = system_shape(lo, hi, tile_off[sys + 1] - tile_off[sys]);
}

constexpr int kRankThreads = 256;        // threads of a rank-pass block
constexpr int kRankChunk = 2048;         // words staged in shared memory at a time

template <int PASS, int G>
__global__ void __launch_bounds__(kRankThreads)
k_rank_pass(const double* __restrict__ pos, int n, const int* sys_of_atom, const int* atom_off,
            const int* tile_off, const int2* shape, const unsigned long long* __restrict__ word,
            unsigned long long* next, const int* sp_in, const uint8_t* ghost_in, const int* zid_in,
            bool mixed, int* perm, double* x, double* y, double* z, float4* xhi, float4* xlo,
            int* sp, uint8_t* ghost, int* local, int* zid)
{
    pdl_wait();
    __shared__ unsigned long long sword[kRankChunk];
    // G lanes per atom a (G = 4, 8 or 32 by the largest system)
    const long long gt = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const int a = (int)(gt / G), lane = (int)(gt % G);
    const bool valid = a < n;
    int sys = 0, a0 = 0, a1 = 0;
    unsigned long long wa = 0;
    if (valid) {
        sys = sys_of_atom[a];
        a0 = atom_off[sys];
        a1 = atom_off[sys + 1];
        wa = word[a];
    }
    // position of a inside its system: the words below its own.  The words of
    // the systems of the block's atoms are staged through shared memory.
    const int afirst = blockIdx.x * (kRankThreads / G);
    const int alast = min(n, afirst + kRankThreads / G) - 1;
    const int r0 = atom_off[sys_of_atom[afirst]], r1 = atom_off[sys_of_atom[alast] + 1];
    int r = 0;
    for (int c0 = r0; c0 < r1; c0 += kRankChunk) {
        const int c1 = min(r1, c0 + kRankChunk);
        __syncthreads();
        for (int k = threadIdx.x; k < c1 - c0; k += kRankThreads) sword[k] = word[c0 + k];
        __syncthreads();
        const int lo = max(a0, c0), hi = min(a1, c1);
        for (int j = lo + lane; j < hi; j += G) r += (int)(sword[j - c0] < wa);
    }
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
    if (!valid || lane != 0) return;
    const int li = a - a0;
    if constexpr (PASS < 2) {
        const unsigned long long group = order_group<PASS>(r, tile_off[sys + 1] - tile_off[sys], shape[sys]);
        next[a] = order_word(group, pos[3 * a + PASS + 1], li);
    } else {
        const int d = a0 + r;
        const double px = pos[3 * a], py = pos[3 * a + 1], pz = pos[3 * a + 2];
        perm[d] = a;
        x[d] = px; y[d] = py; z[d] = pz;
        if (mixed) {
            const Sh32 s = split3(px, py, pz);
            xhi[d] = s.hi;
            xlo[d] = s.lo;
        }
        sp[d] = sp_in[a];
        ghost[d] = ghost_in ? ghost_in[a] : 0;
        local[d] = li;
        if (zid_in) zid[d] = zid_in[a];
    }
}

__global__ void k_gather_sorted(const double* __restrict__ pos, const int* perm, const int* sp_in,
                                const uint8_t* ghost_in, const int* sys_of_atom, const int* atom_off, int n,
                                double* x, double* y, double* z, float4* xhi, float4* xlo, int* sp, uint8_t* ghost,
                                int* local, bool mixed, const int* zid_in, int* zid)
{
    pdl_wait();
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= n) return;
    const int o = perm[a];
    const double px = pos[3 * o], py = pos[3 * o + 1], pz = pos[3 * o + 2];
    x[a] = px; y[a] = py; z[a] = pz;
    if (mixed) {
        const Sh32 s = split3(px, py, pz);
        xhi[a] = s.hi;
        xlo[a] = s.lo;
    }
    sp[a] = sp_in[o];
    ghost[a] = ghost_in ? ghost_in[o] : 0;
    local[a] = o - atom_off[sys_of_atom[o]];
    if (zid_in) zid[a] = zid_in[o];
}

// Bounding sphere (centroid, largest distance) of the tile of sorted atoms
// a0 .. a1 - 1, by one warp.
__device__ __forceinline__ double4 tile_sphere(const double* bx, const double* by, const double* bz, int a0, int a1,
                                               int lane)
{
    const int a = a0 + lane;
    const bool valid = a < a1;
    const double x = valid ? bx[a] : 0.0, y = valid ? by[a] : 0.0, z = valid ? bz[a] : 0.0;
    const double inv = 1.0 / double(a1 - a0);
    const double cx = warp_sum(x) * inv, cy = warp_sum(y) * inv, cz = warp_sum(z) * inv;
    double r = valid ? sqrt((x - cx) * (x - cx) + (y - cy) * (y - cy) + (z - cz) * (z - cz)) : 0.0;
    for (int off = 16; off > 0; off >>= 1) r = fmax(r, __shfl_xor_sync(0xffffffffu, r, off));
    return make_double4(cx, cy, cz, r * (1.0 + 1.0e-12) + 1.0e-12);
}

// Bounding sphere of each tile; one warp per tile.
__global__ void k_tile_bounds(Batch b, const int* tile_sys, int ntiles, double4* tiles)
{
    pdl_wait();
    const int lane = threadIdx.x & 31;
    const int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (t >= ntiles) return;
    const int sys = tile_sys[t];
    const int a0 = b.atom_off[sys] + kTile * (t - b.tile_off[sys]);
    const int a1 = min(a0 + kTile, b.atom_off[sys + 1]);
    const double4 sph = tile_sphere(b.x, b.y, b.z, a0, a1, lane);
    if (lane == 0) tiles[t] = sph;
}

// Ascending bitonic sort of the np (a power of two) words in shared memory by
// the whole block; ends with a barrier.
__device__ __forceinline__ void bitonic_block(unsigned long long* key, int np)
{
    const int half = np >> 1;
    for (int k = 2; k <= np; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int t = threadIdx.x; t < half; t += blockDim.x) {
                const int i = ((t & ~(j - 1)) << 1) | (t & (j - 1));
                const unsigned long long u = key[i], v = key[i + j];
                if ((u > v) == ((i & k) == 0)) { key[i] = v; key[i + j] = u; }
            }
            __syncthreads();
        }
}

// The column order of k_rank_shape / k_rank_pass and the tile spheres of
// k_tile_bounds for systems of at most kOrderBlockMax atoms, one block per
// system and one launch in place of five: the three passes sort the same
// 64-bit words, which are distinct (the local index is their low bits), so a
// sort gives each atom the position its rank does and the results are the
// same bit for bit.  Shared memory: the words of the largest system, padded
// to a power of two.
__global__ void __launch_bounds__(1024)
k_order_block(const double* __restrict__ pos, const int* atom_off, const int* tile_off, const int* sp_in,
              const uint8_t* ghost_in, const int* zid_in, bool mixed, int* perm, double* x, double* y, double* z,
              float4* xhi, float4* xlo, int* sp, uint8_t* ghost, int* local, int* zid, double4* tiles)
{
    pdl_wait();
    extern __shared__ unsigned long long key[];
    __shared__ double red[6][32];
    __shared__ int2 s_shape;
    const int sys = blockIdx.x;
    const int a0 = atom_off[sys], n = atom_off[sys + 1] - a0;
    const int tf = tile_off[sys], nt = tile_off[sys + 1] - tf;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nwarps = blockDim.x >> 5;
    int np = 1;
    while (np < n) np <<= 1;
    // bounding box and the pass-0 words (x), the pad words above all others
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int k = tid; k < np; k += blockDim.x) {
        if (k < n) {
            for (int c = 0; c < 3; c++) {
                const double v = pos[3 * (a0 + k) + c];
                lo[c] = fmin(lo[c], v);
                hi[c] = fmax(hi[c], v);
            }
            key[k] = order_word(0, pos[3 * (a0 + k)], k);
        } else {
            key[k] = ~0ull;
        }
    }
    for (int c = 0; c < 3; c++)
        for (int o = 16; o > 0; o >>= 1) {
            lo[c] = fmin(lo[c], __shfl_xor_sync(0xffffffffu, lo[c], o));
            hi[c] = fmax(hi[c], __shfl_xor_sync(0xffffffffu, hi[c], o));
        }
    if (lane == 0)
        for (int c = 0; c < 3; c++) { red[c][wid] = lo[c]; red[3 + c][wid] = hi[c]; }
    __syncthreads();
    if (tid == 0) {
        for (int w = 1; w < nwarps; w++)
            for (int c = 0; c < 3; c++) {
                lo[c] = fmin(lo[c], red[c][w]);
                hi[c] = fmax(hi[c], red[3 + c][w]);
            }
        s_shape = system_shape(lo, hi, nt);
    }
    bitonic_block(key, np);
    const int2 sh = s_shape;
    constexpr unsigned long long kLocal = (1ull << 20) - 1;
    // pass 0 -> words of pass 1 (slab, y); pass 1 -> words of pass 2 (column, z)
    for (int k = tid; k < n; k += blockDim.x) {
        const int li = (int)(key[k] & kLocal);
        key[k] = order_word(order_group<0>(k, nt, sh), pos[3 * (a0 + li) + 1], li);
    }
    __syncthreads();
    bitonic_block(key, np);
    for (int k = tid; k < n; k += blockDim.x) {
        const int li = (int)(key[k] & kLocal);
        key[k] = order_word(order_group<1>(k, nt, sh), pos[3 * (a0 + li) + 2], li);
    }
    __syncthreads();
    bitonic_block(key, np);
    // the sorted atom arrays (the writes of k_rank_pass<2>)
    for (int k = tid; k < n; k += blockDim.x) {
        const int li = (int)(key[k] & kLocal);
        const int a = a0 + li, d = a0 + k;
        const double px = pos[3 * a], py = pos[3 * a + 1], pz = pos[3 * a + 2];
        perm[d] = a;
        x[d] = px; y[d] = py; z[d] = pz;
        if (mixed) {
            const Sh32 s = split3(px, py, pz);
            xhi[d] = s.hi;
            xlo[d] = s.lo;
        }
        sp[d] = sp_in[a];
        ghost[d] = ghost_in ? ghost_in[a] : 0;
        local[d] = li;
        if (zid_in) zid[d] = zid_in[a];
    }
    __syncthreads();
    for (int t = wid; t < nt; t += nwarps) {
        const int b0 = a0 + kTile * t;
        const double4 sph = tile_sphere(x, y, z, b0, min(b0 + kTile, a0 + n), lane);
        if (lane == 0) tiles[tf + t] = sph;
    }
}

int blocks_for(int n, int warps) { return (n + warps - 1) / warps; }

}  // namespace

size_t sort_temp_bytes(int natoms)
{
    size_t bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, bytes, (const unsigned long long*)nullptr, (unsigned long long*)nullptr,
                                    (const int*)nullptr, (int*)nullptr, natoms);
    return bytes;
}

void launch_spatial_sort(const double* pos, int natoms, const int* sys_of_atom, double cell,
                         unsigned long long* keys_in, unsigned long long* keys_out, int* idx_in, int* perm,
                         void* temp, size_t temp_bytes, cudaStream_t stream)
{
    if (natoms <= 0) return;
    k_morton<<<(natoms + 255) / 256, 256, 0, stream>>>(pos, natoms, sys_of_atom, 1.0 / cell, keys_in, idx_in);
    cub::DeviceRadixSort::SortPairs(temp, temp_bytes, keys_in, keys_out, idx_in, perm, natoms, 0, 64, stream);
}

void launch_rank_order(const double* pos, int natoms, int nsys, int max_atoms, const int* sys_of_atom,
                       const int* atom_off, const int* tile_off, int2* shape, unsigned long long* word_a,
                       unsigned long long* word_b, const int* sp_in, const uint8_t* ghost_in, const int* zid_in, bool mixed, int* perm,
                       double* x, double* y, double* z, float4* xhi, float4* xlo, int* sp, uint8_t* ghost,
                       int* local, int* zid, cudaStream_t stream)
{
    if (natoms <= 0 || nsys <= 0) return;
    // a block of 1024 threads for systems above 256 atoms (two atoms a thread
    // for 2000 atoms instead of sixteen)
    if (max_atoms > 256) launch_pdl(k_rank_shape<1024>, dim3(nsys), dim3(1024), 0, stream, pos, atom_off, tile_off, shape, word_a);
    else launch_pdl(k_rank_shape<kOrderThreads>, dim3(nsys), dim3(kOrderThreads), 0, stream, pos, atom_off, tile_off, shape, word_a);
    // lanes per atom: a whole warp for large systems, groups of 8 or 4 lanes
    // for batches of molecules (a warp would idle on a few dozen words)
    const int g = max_atoms > 512 ? 32 : (max_atoms > 64 ? 8 : 4);
    const unsigned blocks = (unsigned)(((long long)natoms * g + kRankThreads - 1) / kRankThreads);
#define D3_RANK_PASS(P, W_IN, W_OUT)                                                                          \
    do {                                                                                                     \
        if (g == 32) launch_pdl(k_rank_pass<P, 32>, dim3(blocks), dim3(kRankThreads), 0, stream, RANK_ARGS(W_IN, W_OUT)); \
        else if (g == 8) launch_pdl(k_rank_pass<P, 8>, dim3(blocks), dim3(kRankThreads), 0, stream, RANK_ARGS(W_IN, W_OUT)); \
        else launch_pdl(k_rank_pass<P, 4>, dim3(blocks), dim3(kRankThreads), 0, stream, RANK_ARGS(W_IN, W_OUT));  \
    } while (0)
#define RANK_ARGS(W_IN, W_OUT) pos, natoms, sys_of_atom, atom_off, tile_off, shape, W_IN, W_OUT, sp_in, ghost_in, \
                                zid_in, mixed, perm, x, y, z, xhi, xlo, sp, ghost, local, zid
    D3_RANK_PASS(0, word_a, word_b);
    D3_RANK_PASS(1, word_b, word_a);
    D3_RANK_PASS(2, word_a, word_b);
#undef RANK_ARGS
#undef D3_RANK_PASS
}

void launch_order_block(const double* pos, int nsys, int max_atoms, const int* atom_off, const int* tile_off,
                        const int* sp_in, const uint8_t* ghost_in, const int* zid_in, bool mixed, int* perm,
                        double* x, double* y, double* z, float4* xhi, float4* xlo, int* sp, uint8_t* ghost,
                        int* local, int* zid, double4* tiles, cudaStream_t stream)
{
    if (nsys <= 0 || max_atoms <= 0) return;
    int np = 1;
    while (np < max_atoms) np <<= 1;
    const int threads = std::min(1024, std::max(32, np / 2));
    launch_pdl(k_order_block, dim3(nsys), dim3(threads), sizeof(unsigned long long) * np, stream, pos, atom_off,
               tile_off, sp_in, ghost_in, zid_in, mixed, perm, x, y, z, xhi, xlo, sp, ghost, local, zid, tiles);
}

void launch_gather_sorted(const double* pos, const int* perm, const int* sp_in, const uint8_t* ghost_in,
                          const int* sys_of_atom, const int* atom_off, int natoms, double* x, double* y, double* z,
                          float4* xhi, float4* xlo, int* sp, uint8_t* ghost, int* local, bool mixed,
                          cudaStream_t stream, const int* zid_in, int* zid)
{
    if (natoms <= 0) return;
    launch_pdl(k_gather_sorted, dim3((natoms + 255) / 256), dim3(256), 0, stream, pos, perm, sp_in, ghost_in, sys_of_atom, atom_off,
                                                              natoms, x, y, z, xhi, xlo, sp, ghost, local, mixed,
                                                              zid_in, zid);
}

void launch_tile_bounds(const Batch& b, const int* tile_sys, int ntiles, double4* tiles, cudaStream_t stream)
{
    if (ntiles <= 0) return;
    launch_pdl(k_tile_bounds, dim3((ntiles + 7) / 8), dim3(256), 0, stream, b, tile_sys, ntiles, tiles);
}

// Atoms per block of the pair sweeps: 4 or 8 warps (one atom per warp).
#define D3_PAIR_LAUNCH(KERNEL, ...)                                                                   \
    do {                                                                                             \
        if (c.pair_warps == 4) KERNEL<4, __VA_ARGS__><<<blocks_for(b.natoms, 4), 128, 0, stream>>>ARGS; \
        else KERNEL<8, __VA_ARGS__><<<blocks_for(b.natoms, 8), 256, 0, stream>>>ARGS;                  \
    } while (0)

void launch_coordination_number_tiled(const Batch& b, const Species& s, const Config& c, const Partition& p,
                                      const Work& w, cudaStream_t stream)
{
#define ARGS (b, s, c, p, w)
    if (c.mixed) D3_PAIR_LAUNCH(k_cn_tiled, float);
    else D3_PAIR_LAUNCH(k_cn_tiled, double);
#undef ARGS
}

void launch_two_body_tiled(const Batch& b, const Species& s, const Damp& d, const Config& c, const Partition& p,
                           const Work& w, cudaStream_t stream)
{
#define ARGS (b, s, d, c, p, w)
    if (d.kind == kRational) {
        if (c.mixed) D3_PAIR_LAUNCH(k_two_body_tiled, float, kRational);
        else D3_PAIR_LAUNCH(k_two_body_tiled, double, kRational);
    } else {
        if (c.mixed) D3_PAIR_LAUNCH(k_two_body_tiled, float, kZero);
        else D3_PAIR_LAUNCH(k_two_body_tiled, double, kZero);
    }
#undef ARGS
}

void launch_cn_chain_rule_tiled(const Batch& b, const Species& s, const Config& c, const Partition& p,
                                const Work& w, cudaStream_t stream)
{
#define ARGS (b, s, c, p, w)
    if (c.mixed) D3_PAIR_LAUNCH(k_chain_tiled, float);
    else D3_PAIR_LAUNCH(k_chain_tiled, double);
#undef ARGS
}

#undef D3_PAIR_LAUNCH

}  // namespace d3
