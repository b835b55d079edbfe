// CUDA kernels of the D3 dispersion hot path for sm_100a.
//
// Layout: one warp per atom i.  The warp keeps the positions of atom i shifted
// by a chunk of lattice translations, y(T) = x_i - T, in shared memory, and
// sweeps the atoms j of the same system 32 at a time (one j per lane).  Every
// atom accumulates only its own energy, dE/dCN, gradient and virial share
// (a full neighbour sum instead of the reference's j <= i half sum, which
// needs no atomics and gives bit-reproducible results); the warp reduces the
// lanes in a fixed order.
//
// Precision: the FP64 form does all arithmetic in double.  The mixed form
// forms displacements from double-float (head + tail) coordinates, evaluates
// the pair terms in FP32 and accumulates in FP64.
#include <algorithm>
#include <cfloat>
#include <cstdint>

#include "d3_device.cuh"
#include "d3_weights.cuh"

namespace d3 {

namespace {

constexpr int kWarpsPerBlock = 8;
constexpr int kDirectWarps = 4;       // warps per atom of the small-system (input order) kernels
constexpr int kThreads = 32 * kWarpsPerBlock;
constexpr int kImgChunk = 128;        // images staged per warp and pass
constexpr double kKcn = 16.0;         // ncoord.f90:31
constexpr double kWf = 4.0;           // model.f90:80

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    return v;
}

__device__ __forceinline__ bool owns_pair(const Partition& p, int i, int j)
{
    // partition.f90:127-147 on zero-based system-local indices
    if (p.nparts <= 1) return true;
    long long hi = i > j ? i : j, lo = i > j ? j : i;
    long long idx = hi * (hi + 1) / 2 + lo;
    return idx % p.nparts == p.part;
}

template <class R>
__device__ __forceinline__ void smooth_cutoff(R r, R cutoff, R width, R& sw, R& dswdr)
{
    // cutoff.f90:73-99
    if (width <= R(0) || width >= cutoff) { sw = R(1); dswdr = R(0); return; }
    R inner = cutoff - width;
    if (r <= inner) { sw = R(1); dswdr = R(0); }
    else if (r >= cutoff) { sw = R(0); dswdr = R(0); }
    else {
        R x = (cutoff - r) / width;
        sw = x * x * x * (R(10) + x * (R(-15) + R(6) * x));
        dswdr = R(-30) * x * x * (R(1) - x) * (R(1) - x) / width;
    }
}

// Shifted position of atom i for one image, in the representation of the form.
struct Shift64 { double x, y, z; };
struct Shift32 { float4 hi, lo; };

template <class R> struct ShiftOf;
template <> struct ShiftOf<double> { using type = Shift64; };
template <> struct ShiftOf<float> { using type = Shift32; };

__device__ __forceinline__ Shift32 split_shift(double x, double y, double z)
{
    Shift32 s;
    s.hi = make_float4(__double2float_rn(x), __double2float_rn(y), __double2float_rn(z), 0.f);
    s.lo = make_float4(__double2float_rn(x - (double)s.hi.x), __double2float_rn(y - (double)s.hi.y),
                       __double2float_rn(z - (double)s.hi.z), 0.f);
    return s;
}

// Displacement y(T) - x_j in the working precision.
__device__ __forceinline__ void displacement(const Shift64& s, double xj, double yj, double zj,
                                             float4, float4, double& vx, double& vy, double& vz)
{
    vx = s.x - xj; vy = s.y - yj; vz = s.z - zj;
}

__device__ __forceinline__ void displacement(const Shift32& s, double, double, double,
                                             float4 hj, float4 lj, float& vx, float& vy, float& vz)
{
    vx = (s.hi.x - hj.x) + (s.lo.x - lj.x);
    vy = (s.hi.y - hj.y) + (s.lo.y - lj.y);
    vz = (s.hi.z - hj.z) + (s.lo.z - lj.z);
}

// Stage y(T) = x_i - T for images [t0, t0 + nt) of this warp into shared memory.
template <class R>
__device__ __forceinline__ void stage_images(typename ShiftOf<R>::type* buf, const double* img,
                                             int t0, int nt, double xi, double yi, double zi, int lane)
{
    for (int k = lane; k < nt; k += 32) {
        const double tx = __ldg(img + 3 * (t0 + k) + 0);
        const double ty = __ldg(img + 3 * (t0 + k) + 1);
        const double tz = __ldg(img + 3 * (t0 + k) + 2);
        if constexpr (sizeof(R) == 8) {
            buf[k] = Shift64{xi - tx, yi - ty, zi - tz};
        } else {
            buf[k] = split_shift(xi - tx, yi - ty, zi - tz);
        }
    }
    __syncwarp();
}

template <class R>
__device__ __forceinline__ R rexp(R x) { if constexpr (sizeof(R) == 8) return exp(x); else return expf(x); }
template <class R>
__device__ __forceinline__ R rsqrt_(R x) { if constexpr (sizeof(R) == 8) return sqrt(x); else return sqrtf(x); }
template <class R>
__device__ __forceinline__ R rinv_sqrt(R x) { if constexpr (sizeof(R) == 8) return rsqrt(x); else return rsqrtf(x); }
template <class R>
__device__ __forceinline__ R rpow(R x, R a) { if constexpr (sizeof(R) == 8) return pow(x, a); else return powf(x, a); }

// ------------------------------------------------------------ positions ----

__global__ void k_split_positions(const double* __restrict__ pos, int n, double* x, double* y,
                                  double* z, float4* xhi, float4* xlo, bool mixed)
{
    pdl_wait();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double px = pos[3 * i + 0], py = pos[3 * i + 1], pz = pos[3 * i + 2];
    x[i] = px; y[i] = py; z[i] = pz;
    if (mixed) {
        Shift32 s = split_shift(px, py, pz);
        xhi[i] = s.hi;
        xlo[i] = s.lo;
    }
}

// Warps per atom of the warp-per-atom kernels: warp g of an atom takes its
// partner blocks g, g + G, ...; the warps' sums meet in shared memory and the
// atom's first warp adds them in warp order (a fixed order).  Returns whether
// this warp holds the atom's totals in v (all lanes).
template <int G, int NV>
__device__ __forceinline__ bool combine_warps(double (&v)[NV], double (*part)[16], int wib, int lane, bool active)
{
    static_assert(NV <= 16, "values per atom");
    if constexpr (G == 1) {
        return active;
    } else {
        if (lane == 0)
            for (int k = 0; k < NV; k++) part[wib][k] = v[k];
        __syncthreads();
        if (!active || wib % G != 0) return false;
        for (int k = 0; k < NV; k++) {
            double t = 0.0;
            for (int q = 0; q < G; q++) t += part[wib + q][k];
            v[k] = t;
        }
        return true;
    }
}

// ----------------------------------------------------- coordination number --

// CN_i = sum_{j,T} 1/(1 + exp(-kcn (rc/r - 1))) for 1e-12 <= r^2 <= cutoff^2
// (get_partitioned_coordination_number, ncoord.f90:86-144).  W (atoms in
// input order): the positions come from the input array and the warp writes
// its atom's position arrays for the later kernels, then goes on with the
// atom's reference weights and, into UV, its species vectors (atom_weights),
// in place of separate gather, weight and vector kernels.
template <class R, bool W, int G>
__global__ void __launch_bounds__(kThreads) k_coordination_number(Batch b, Species s, Config c,
                                                                  Partition p, Work w, R* UV, InputPositions in)
{
    pdl_wait();
    using Sh = typename ShiftOf<R>::type;
    __shared__ Sh sbuf[kWarpsPerBlock][kImgChunk];
    __shared__ double part[kWarpsPerBlock][16];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, g = wib % G;
    const int i0 = blockIdx.x * (kWarpsPerBlock / G) + wib / G;
    const bool active = i0 < b.natoms;
    const int i = active ? i0 : b.natoms - 1;
    const int sys = b.sys_of_atom[i];
    const int j0 = b.atom_off[sys], j1 = b.atom_off[sys + 1];
    const int t0 = b.img_off[kImgCN * (b.nsys + 1) + sys], t1 = b.img_off[kImgCN * (b.nsys + 1) + sys + 1];
    const double xi = W ? in.pos[3 * i] : b.x[i], yi = W ? in.pos[3 * i + 1] : b.y[i], zi = W ? in.pos[3 * i + 2] : b.z[i];
    const double rci = s.rcov[b.sp[i]];
    const int li = b.local[i];
    const R cut2 = R(c.cut_cn * c.cut_cn);
    double acc = 0.0;
    unsigned long long nterm = 0;
    for (int tc = t0; tc < t1; tc += kImgChunk) {
        const int nt = min(kImgChunk, t1 - tc);
        stage_images<R>(sbuf[wib], b.img, tc, nt, xi, yi, zi, lane);
        for (int jb = j0 + 32 * g; active && jb < j1; jb += 32 * G) {
            const int j = jb + lane;
            const bool valid = j < j1 && (!c.cn_partitioned || owns_pair(p, li, j - j0));
            const int jj = valid ? j : j0;
            double xj, yj, zj;
            float4 hj = make_float4(0, 0, 0, 0), lj = hj;
            if constexpr (W) {
                xj = in.pos[3 * jj]; yj = in.pos[3 * jj + 1]; zj = in.pos[3 * jj + 2];
                if constexpr (sizeof(R) == 4) {
                    const Shift32 sj = split_shift(xj, yj, zj);
                    hj = sj.hi; lj = sj.lo;
                }
            } else {
                xj = b.x[jj]; yj = b.y[jj]; zj = b.z[jj];
                if constexpr (sizeof(R) == 4) { hj = b.xhi[jj]; lj = b.xlo[jj]; }
            }
            const R rc = R(rci + s.rcov[b.sp[jj]]);
            for (int k = 0; k < nt; k++) {
                R vx, vy, vz;
                displacement(sbuf[wib][k], xj, yj, zj, hj, lj, vx, vy, vz);
                const R r2 = vx * vx + vy * vy + vz * vz;
                if (!valid || r2 > cut2 || r2 < R(1.0e-12)) continue;
                const R cf = R(1) / (R(1) + rexp(-R(kKcn) * (rc * rinv_sqrt(r2) - R(1))));
                acc += double(cf);
                nterm += (jj <= i);
            }
        }
        __syncwarp();
    }
    acc = warp_sum(acc);
    if (w.counts && active) {
        for (int off = 16; off > 0; off >>= 1) nterm += __shfl_xor_sync(0xffffffffu, nterm, off);
        if (lane == 0) atomicAdd(w.counts + 2, nterm);
    }
    double v[1] = {acc};
    if (!combine_warps<G, 1>(v, part, wib, lane, active)) return;
    acc = v[0];
    if (lane == 0) w.cn[i] = acc;
    if (W) {
        if (lane == 0) {
            in.x[i] = xi; in.y[i] = yi; in.z[i] = zi;
            if (c.mixed) {
                const Shift32 si = split_shift(xi, yi, zi);
                in.xhi[i] = si.hi;
                in.xlo[i] = si.lo;
            }
        }
        atom_weights<R>(b, s, c, w, i, acc, lane, UV);
    }
}

// ---------------------------------------------------------------- weights --

// Gaussian reference weights and their CN derivative with the reference's
// NaN/Inf fallback (weight_references, model.f90:201-324), always FP64.
__global__ void k_weights(Batch b, Species s, Config c, Work w)
{
    pdl_wait();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= b.natoms) return;
    const int sp = b.sp[i];
    const int nref = s.nref[sp];
    const double* cnref = s.refcn + sp * kMaxRef;
    const double cn = w.cn[i];
    const double wf2 = 2 * kWf;
    double gwt[kMaxRef];
    double norm = 0.0, dnorm = 0.0;
    double maxcn = cnref[0];
    for (int r = 0; r < nref; r++) {
        const double d = cn - cnref[r];
        const double g = exp(-kWf * d * d);
        gwt[r] = g;
        norm = norm + g;
        dnorm = dnorm + wf2 * (cnref[r] - cn) * g;
        maxcn = fmax(maxcn, cnref[r]);
    }
    norm = 1.0 / norm;
    for (int r = 0; r < kMaxRef; r++) {
        double gwk = 0.0, dgwk = 0.0;
        if (r < nref) {
            const double expw = gwt[r];
            const double expd = wf2 * (cnref[r] - cn) * expw;
            gwk = expw * norm;
            if (isnan(gwk) || isinf(gwk)) gwk = (maxcn == cnref[r]) ? 1.0 : 0.0;
            dgwk = expd * norm - expw * dnorm * (norm * norm);
            if (isnan(dgwk) || isinf(dgwk)) dgwk = 0.0;
        }
        w.gw[i * kMaxRef + r] = gwk;
        w.dgw[i * kMaxRef + r] = dgwk;
        if (c.mixed) {
            w.gwf[i * kMaxRef + r] = float(gwk);
            w.dgwf[i * kMaxRef + r] = float(dgwk);
        }
    }
}

// C6_ij and its CN derivatives from the reference weights
// (get_atomic_c6, model.f90:432-461).
template <class R>
__device__ __forceinline__ void atomic_c6(const Species& s, int nid, int si, int sj, int nri, int nrj,
                                          const R* gwi, const R* dgwi, const R* gwj, const R* dgwj,
                                          R& c6, R& dc6i, R& dc6j)
{
    const int base = (si * nid + sj) * kMaxRef * kMaxRef;
    c6 = R(0); dc6i = R(0); dc6j = R(0);
    for (int ir = 0; ir < nri; ir++) {
        R a = R(0), bj = R(0);
        for (int jr = 0; jr < nrj; jr++) {
            R ref;
            if constexpr (sizeof(R) == 8) ref = __ldg(s.c6ref + base + ir * kMaxRef + jr);
            else ref = __ldg(s.c6ref_f + base + ir * kMaxRef + jr);
            a += gwj[jr] * ref;
            bj += dgwj[jr] * ref;
        }
        c6 += gwi[ir] * a;
        dc6i += dgwi[ir] * a;
        dc6j += gwi[ir] * bj;
    }
}

// ---------------------------------------------------------------- two-body --

// Rational (rational.f90:378-514) and zero (zero.f90:409-553) damped pair sum
// with energy, dE/dCN, gradient, virial and optional parameter derivatives.
template <class R, int DAMP, int G>
__global__ void __launch_bounds__(kThreads) k_two_body(Batch b, Species s, Damp d, Config c,
                                                       Partition p, Work w, const R* UV)
{
    pdl_wait();
    using Sh = typename ShiftOf<R>::type;
    __shared__ Sh sbuf[kWarpsPerBlock][kImgChunk];
    __shared__ double part[kWarpsPerBlock][16];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, g = wib % G;
    const int i0 = blockIdx.x * (kWarpsPerBlock / G) + wib / G;
    const bool active = i0 < b.natoms;
    const int i = active ? i0 : b.natoms - 1;
    const int sys = b.sys_of_atom[i];
    const int j0 = b.atom_off[sys], j1 = b.atom_off[sys + 1];
    const int t0 = b.img_off[kImgDisp2 * (b.nsys + 1) + sys];
    const int t1 = b.img_off[kImgDisp2 * (b.nsys + 1) + sys + 1];
    const double xi = b.x[i], yi = b.y[i], zi = b.z[i];
    const int si = b.sp[i], nid = b.nid;
    const int nri = s.nref[si];
    const int li = b.local[i];
    const bool gi = b.ghost && b.ghost[i];
    R gwi[kMaxRef], dgwi[kMaxRef];
    for (int r = 0; r < kMaxRef; r++) {
        if constexpr (sizeof(R) == 8) { gwi[r] = w.gw[i * kMaxRef + r]; dgwi[r] = w.dgw[i * kMaxRef + r]; }
        else { gwi[r] = w.gwf[i * kMaxRef + r]; dgwi[r] = w.dgwf[i * kMaxRef + r]; }
    }
    const R cutoff = R(c.cut2), cut2 = R(c.cut2 * c.cut2), width = R(c.width2);
    const bool smooth = c.width2 > 0.0 && c.width2 < c.cut2;
    const R s6 = R(d.s6), s8 = R(d.s8);
    const R alp6 = R(d.alp), alp8 = R(d.alp + 2.0);
    double e = 0, de = 0, gx = 0, gy = 0, gz = 0;
    double sxx = 0, syy = 0, szz = 0, sxy = 0, sxz = 0, syz = 0;
    double pg0 = 0, pg1 = 0, pg2 = 0, pg3 = 0;
    unsigned long long nterm = 0;
    for (int tc = t0; tc < t1; tc += kImgChunk) {
        const int nt = min(kImgChunk, t1 - tc);
        stage_images<R>(sbuf[wib], b.img, tc, nt, xi, yi, zi, lane);
        for (int jb = j0 + 32 * g; active && jb < j1; jb += 32 * G) {
            const int j = jb + lane;
            const bool valid = j < j1 && owns_pair(p, li, j - j0);
            const int jj = j < j1 ? j : j0;
            const double xj = b.x[jj], yj = b.y[jj], zj = b.z[jj];
            float4 hj = make_float4(0, 0, 0, 0), lj = hj;
            if constexpr (sizeof(R) == 4) { hj = b.xhi[jj]; lj = b.xlo[jj]; }
            const int sj = b.sp[jj];
            const int nrj = s.nref[sj];
            R c6 = R(0), dc6i = R(0), dc6j = R(0);
            if (UV && valid && !gi) {
                // from the species vectors of j for i's species (zero for a ghost j), vector loads
                R u[2 * kRefPad];
                const R* up = UV + ((size_t)jj * nid + si) * (2 * kRefPad);
                if constexpr (sizeof(R) == 4) {
#pragma unroll
                    for (int q = 0; q < kRefPad / 2; q++) {
                        const float4 v4 = __ldg(reinterpret_cast<const float4*>(up) + q);
                        u[4 * q] = v4.x; u[4 * q + 1] = v4.y; u[4 * q + 2] = v4.z; u[4 * q + 3] = v4.w;
                    }
                } else {
#pragma unroll
                    for (int q = 0; q < kRefPad; q++) {
                        const double2 v2 = __ldg(reinterpret_cast<const double2*>(up) + q);
                        u[2 * q] = v2.x; u[2 * q + 1] = v2.y;
                    }
                }
#pragma unroll
                for (int r = 0; r < kMaxRef; r++) {
                    c6 += gwi[r] * u[r];
                    dc6i += dgwi[r] * u[r];
                    dc6j += gwi[r] * u[kRefPad + r];
                }
            } else if (valid && !gi && !(b.ghost && b.ghost[jj])) {
                R gwj[kMaxRef], dgwj[kMaxRef];
                for (int r = 0; r < kMaxRef; r++) {
                    if constexpr (sizeof(R) == 8) { gwj[r] = w.gw[jj * kMaxRef + r]; dgwj[r] = w.dgw[jj * kMaxRef + r]; }
                    else { gwj[r] = w.gwf[jj * kMaxRef + r]; dgwj[r] = w.dgwf[jj * kMaxRef + r]; }
                }
                atomic_c6<R>(s, nid, si, sj, nri, nrj, gwi, dgwi, gwj, dgwj, c6, dc6i, dc6j);
            }
            const double2* pr = reinterpret_cast<const double2*>(s.pair + kPairSlots * (si * nid + sj));
            const double2 p01 = __ldg(pr), p23 = __ldg(pr + 1), p45 = __ldg(pr + 2);
            const R rrij = R(p01.x);
            const R q1 = R(p01.y), q2 = R(p23.x), q3 = R(p23.y);
            const R q4 = R(p45.x);
            for (int k = 0; k < nt; k++) {
                R vx, vy, vz;
                displacement(sbuf[wib][k], xj, yj, zj, hj, lj, vx, vy, vz);
                const R r2 = vx * vx + vy * vy + vz * vz;
                if (!valid || r2 > cut2 || r2 < R(DBL_EPSILON)) continue;
                nterm += (jj <= i);   // the reference's (i, j <= i, T) count
                R sw = R(1), dswdr = R(0), r1 = R(0);
                if (smooth) { r1 = rsqrt_(r2); smooth_cutoff<R>(r1, cutoff, width, sw, dswdr); }
                R edisp0, gdisp0, e6, e8, dpa = R(0), dpb = R(0);
                if constexpr (DAMP == kRational) {
                    // q1 = R0^6, q2 = R0^8, q3 = R0 = a1 sqrt(rrij) + a2, q4 = sqrt(rrij)
                    const R r4 = r2 * r2;
                    // one reciprocal for both denominators
                    const R a6 = r4 * r2 + q1, a8 = r4 * r4 + q2;
                    const R inv = R(1) / (a6 * a8);
                    const R t6 = a8 * inv;
                    const R t8 = a6 * inv;
                    const R d6 = R(-6) * r4 * t6 * t6;
                    const R d8 = R(-8) * r4 * r2 * t8 * t8;
                    e6 = t6; e8 = rrij * t8;
                    edisp0 = s6 * t6 + s8 * rrij * t8;
                    gdisp0 = s6 * d6 + s8 * rrij * d8;
                    if (c.param_grad) {
                        // dt6/dR0 = -6 R0^5 t6^2, dt8/dR0 = -8 R0^7 t8^2; dR0/da1 = sqrt(rrij)
                        const R r05 = q1 / q3, r07 = q2 / q3;
                        const R dedr0 = s6 * R(-6) * r05 * t6 * t6 + s8 * rrij * R(-8) * r07 * t8 * t8;
                        dpa = dedr0 * q4;
                        dpb = dedr0;
                    }
                } else {
                    // q1 = rs6 * R0, q2 = rs8 * R0
                    if (!smooth) r1 = rsqrt_(r2);
                    const R r6 = r2 * r2 * r2;
                    const R r8 = r6 * r2;
                    const R t6 = rpow<R>(q1 / r1, alp6);
                    const R t8 = rpow<R>(q2 / r1, alp8);
                    const R f6 = R(1) / (R(1) + R(6) * t6);
                    const R f8 = R(1) / (R(1) + R(6) * t8);
                    const R d6 = R(-6) * f6 / r2 + R(6) * alp6 * t6 * (f6 * f6) / r2;
                    const R d8 = R(-8) * f8 / r2 + R(6) * alp8 * t8 * (f8 * f8) / r2;
                    e6 = f6 / r6; e8 = rrij * f8 / r8;
                    edisp0 = s6 * f6 / r6 + s8 * rrij * f8 / r8;
                    gdisp0 = s6 * d6 / r6 + s8 * rrij * d8 / r8;
                    if (c.param_grad) {
                        // t = (rs R0 / r)^alp: dt/drs = alp t / rs, df/dt = -6 f^2
                        dpa = d.rs6 != 0.0 ? s6 / r6 * R(-6) * f6 * f6 * alp6 * t6 / R(d.rs6) : R(0);
                        dpb = d.rs8 != 0.0 ? s8 * rrij / r8 * R(-6) * f8 * f8 * alp8 * t8 / R(d.rs8) : R(0);
                    }
                }
                const R edisp = sw * edisp0;
                e += double(-c6 * edisp * R(0.5));
                de -= double(dc6i * edisp);
                if (c.param_grad) {
                    const R hc = R(-0.5) * c6 * sw;
                    pg0 += double(hc * e6);
                    pg1 += double(hc * e8);
                    pg2 += double(hc * dpa);
                    pg3 += double(hc * dpb);
                }
                if (!c.grad) continue;
                R gdisp = sw * gdisp0;
                if (smooth) gdisp += dswdr * edisp0 / r1;
                const R f = -c6 * gdisp;
                const R dgx = f * vx, dgy = f * vy, dgz = f * vz;
                if (jj != i) { gx += double(dgx); gy += double(dgy); gz += double(dgz); }
                sxx += double(R(0.5) * dgx * vx); syy += double(R(0.5) * dgy * vy);
                szz += double(R(0.5) * dgz * vz); sxy += double(R(0.5) * dgx * vy);
                sxz += double(R(0.5) * dgx * vz); syz += double(R(0.5) * dgy * vz);
            }
        }
        __syncwarp();
    }
    if (w.counts && active) {
        for (int off = 16; off > 0; off >>= 1) nterm += __shfl_xor_sync(0xffffffffu, nterm, off);
        if (lane == 0) atomicAdd(w.counts + 0, nterm);
    }
    double v[15] = {e, de, gx, gy, gz, sxx, syy, szz, sxy, sxz, syz, pg0, pg1, pg2, pg3};
    for (int k = 0; k < 15; k++) v[k] = warp_sum(v[k]);
    if (!combine_warps<G, 15>(v, part, wib, lane, active)) return;
    e = v[0]; de = v[1]; gx = v[2]; gy = v[3]; gz = v[4];
    sxx = v[5]; syy = v[6]; szz = v[7]; sxy = v[8]; sxz = v[9]; syz = v[10];
    pg0 = v[11]; pg1 = v[12]; pg2 = v[13]; pg3 = v[14];
    if (lane == 0) w.e_atom[i] = e;
    if (c.grad) {
        if (lane == 0) {
            w.dEdcn[i] = de;
            w.grad[3 * i + 0] = gx; w.grad[3 * i + 1] = gy; w.grad[3 * i + 2] = gz;
            double* sg = w.sig_atom + kSigma * i;
            sg[0] = sxx; sg[1] = syy; sg[2] = szz; sg[3] = sxy; sg[4] = sxz; sg[5] = syz;
        }
    }
    if (c.param_grad) {
        if (lane == 0) {
            double* pg = w.pg_atom + kParamGrad * i;
            pg[0] = pg0; pg[1] = pg1; pg[2] = pg2; pg[3] = pg3;
        }
    }
}

// ------------------------------------------------------------- chain rule --

// gradient += dE/dCN dCN/dR, sigma += dE/dCN dCN/deps
// (add_coordination_number_derivs, ncoord.f90:152-228).
template <class R, int G>
__global__ void __launch_bounds__(kThreads) k_cn_chain(Batch b, Species s, Config c, Partition p, Work w)
{
    pdl_wait();
    using Sh = typename ShiftOf<R>::type;
    __shared__ Sh sbuf[kWarpsPerBlock][kImgChunk];
    __shared__ double part[kWarpsPerBlock][16];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, g = wib % G;
    const int i0 = blockIdx.x * (kWarpsPerBlock / G) + wib / G;
    const bool active = i0 < b.natoms;
    const int i = active ? i0 : b.natoms - 1;
    const int sys = b.sys_of_atom[i];
    const int j0 = b.atom_off[sys], j1 = b.atom_off[sys + 1];
    const int t0 = b.img_off[kImgCN * (b.nsys + 1) + sys], t1 = b.img_off[kImgCN * (b.nsys + 1) + sys + 1];
    const double xi = b.x[i], yi = b.y[i], zi = b.z[i];
    const double rci = s.rcov[b.sp[i]];
    const double dei = w.dEdcn[i];
    const int li = b.local[i];
    const R cut2 = R(c.cut_cn * c.cut_cn);
    double gx = 0, gy = 0, gz = 0, sxx = 0, syy = 0, szz = 0, sxy = 0, sxz = 0, syz = 0;
    for (int tc = t0; tc < t1; tc += kImgChunk) {
        const int nt = min(kImgChunk, t1 - tc);
        stage_images<R>(sbuf[wib], b.img, tc, nt, xi, yi, zi, lane);
        for (int jb = j0 + 32 * g; active && jb < j1; jb += 32 * G) {
            const int j = jb + lane;
            const bool valid = j < j1 && (!c.cn_partitioned || owns_pair(p, li, j - j0));
            const int jj = j < j1 ? j : j0;
            const double xj = b.x[jj], yj = b.y[jj], zj = b.z[jj];
            float4 hj = make_float4(0, 0, 0, 0), lj = hj;
            if constexpr (sizeof(R) == 4) { hj = b.xhi[jj]; lj = b.xlo[jj]; }
            const R rc = R(rci + s.rcov[b.sp[jj]]);
            // 0.5 (dEdcn_i + dEdcn_j) weights the virial share of this atom;
            // the full (i, j) sum counts every pair twice, self images once per T
            const R dsum = R(dei + w.dEdcn[jj]);
            for (int k = 0; k < nt; k++) {
                R vx, vy, vz;
                displacement(sbuf[wib][k], xj, yj, zj, hj, lj, vx, vy, vz);
                const R r2 = vx * vx + vy * vy + vz * vz;
                if (!valid || r2 > cut2 || r2 < R(1.0e-12)) continue;
                const R ir = rinv_sqrt(r2);
                const R expterm = rexp(-R(kKcn) * (rc * ir - R(1)));
                const R cf = R(1) / (R(1) + expterm);
                // dcf / r with dcf = -cf (1 - cf) kcn rc / r^2 (ncoord.f90:198-201)
                const R f = -cf * (R(1) - cf) * R(kKcn) * rc * (ir * ir * ir) * dsum;
                const R cx = f * vx, cy = f * vy, cz = f * vz;
                if (jj != i) { gx += double(cx); gy += double(cy); gz += double(cz); }
                sxx += double(R(0.5) * cx * vx); syy += double(R(0.5) * cy * vy);
                szz += double(R(0.5) * cz * vz); sxy += double(R(0.5) * cx * vy);
                sxz += double(R(0.5) * cx * vz); syz += double(R(0.5) * cy * vz);
            }
        }
        __syncwarp();
    }
    double v[9] = {gx, gy, gz, sxx, syy, szz, sxy, sxz, syz};
    for (int k = 0; k < 9; k++) v[k] = warp_sum(v[k]);
    if (!combine_warps<G, 9>(v, part, wib, lane, active)) return;
    gx = v[0]; gy = v[1]; gz = v[2]; sxx = v[3]; syy = v[4]; szz = v[5]; sxy = v[6]; sxz = v[7]; syz = v[8];
    if (lane == 0) {
        w.grad[3 * i + 0] += gx; w.grad[3 * i + 1] += gy; w.grad[3 * i + 2] += gz;
        double* sg = w.sig_atom + kSigma * i;
        sg[0] += sxx; sg[1] += syy; sg[2] += szz; sg[3] += sxy; sg[4] += sxz; sg[5] += syz;
    }
}

// ------------------------------------------------------------- reductions --

// Per-system sums of the atom energies, virial shares and parameter
// derivatives in a fixed order (one block per system).
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK)
k_reduce_systems(Batch b, Config c, Work w, double* energies, double* sigma9, double* param_grad, double* grad_out)
{
    pdl_wait();
    constexpr int kVals = 1 + kSigma + kParamGrad;
    __shared__ double red[kVals][BLOCK / 32];
    const int sys = blockIdx.x;
    const int a0 = b.atom_off[sys], a1 = b.atom_off[sys + 1];
    double v[kVals];
    for (int k = 0; k < kVals; k++) v[k] = 0.0;
    for (int a = a0 + threadIdx.x; a < a1; a += BLOCK) {
        v[0] += w.e_atom[a] + (w.e3_atom ? w.e3_atom[a] : 0.0);
        if (c.grad)
            for (int k = 0; k < kSigma; k++)
                v[1 + k] += w.sig_atom[kSigma * a + k] + (w.sig3_atom ? w.sig3_atom[kSigma * a + k] : 0.0);
        if (c.param_grad && w.pg_atom)
            for (int k = 0; k < kParamGrad - 1; k++) v[1 + kSigma + k] += w.pg_atom[kParamGrad * a + k];
        if (c.param_grad && w.e3_pg) v[kSigma + kParamGrad] += w.e3_pg[a] * w.pg_s9_scale;
        if (c.grad && grad_out) {
            const int o = b.perm ? b.perm[a] : a;
            for (int k = 0; k < 3; k++) grad_out[3 * o + k] = w.grad[3 * a + k];
        }
    }
    // warp sums, then the warps' sums in warp order (a fixed order)
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int k = 0; k < kVals; k++) {
        double x = v[k];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == 0) red[k][wid] = x;
    }
    __syncthreads();
    if (wid != 0) return;
    double tot = 0.0;
    if (lane < kVals)
        for (int q = 0; q < BLOCK / 32; q++) tot += red[lane][q];
    // lane k holds value k
    if (lane == 0 && energies) energies[sys] = tot;
    if (c.grad && sigma9 && lane >= 1 && lane <= kSigma) {
        // Fortran sigma(3,3): element (a, b) at a + 3 b; symmetric; packed xx yy zz xy xz yz
        constexpr int kAt[kSigma][2] = {{0, 0}, {4, 4}, {8, 8}, {1, 3}, {2, 6}, {5, 7}};
        double* o = sigma9 + 9 * sys;
        o[kAt[lane - 1][0]] = tot;
        o[kAt[lane - 1][1]] = tot;
    }
    if (c.param_grad && param_grad && lane > kSigma && lane < kVals) param_grad[kParamGrad * sys + lane - 1 - kSigma] = tot;
}

// Dependent-FMA throughput probe: 8 independent chains per thread, used to
// measure the FP64/FP32 pipe peak the roofline is quoted against.
template <class T>
__global__ void __launch_bounds__(256) k_fma_peak(T* out, int iters)
{
    T x[8];
#pragma unroll
    for (int k = 0; k < 8; k++) x[k] = T(1) + T(threadIdx.x + k) * T(1e-7);
    const T b = T(0.9999999), c = T(1e-7);
    for (int it = 0; it < iters; it++) {
#pragma unroll
        for (int k = 0; k < 8; k++) x[k] = fma(x[k], b, c);
    }
    T sum = T(0);
#pragma unroll
    for (int k = 0; k < 8; k++) sum += x[k];
    if (sum == T(-1)) out[blockIdx.x] = sum;  // never true; keeps the chains live
}

int blocks_for_atoms(int n, int warps_per_atom = 1)
{
    const int per_block = kWarpsPerBlock / warps_per_atom;
    return (n + per_block - 1) / per_block;
}

}  // namespace

double measure_fma_peak(bool fp64)
{
    // returns TFLOP/s of fused multiply-adds (2 flops each) over a ~0.1 s launch
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int blocks = sms * 16, threads = 256;
    const int iters = fp64 ? 4096 : 8192;
    void* out = nullptr;
    cudaMalloc(&out, sizeof(double) * blocks);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double best = 0.0;
    for (int rep = 0; rep < 5; rep++) {
        cudaEventRecord(e0);
        if (fp64) k_fma_peak<double><<<blocks, threads>>>((double*)out, iters);
        else k_fma_peak<float><<<blocks, threads>>>((float*)out, iters);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        const double flops = 2.0 * 8.0 * iters * (double)blocks * threads;
        if (ms > 0) best = std::max(best, flops / (ms * 1e-3) / 1e12);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    return best;
}

void launch_split_positions(const double* pos, int natoms, double* x, double* y, double* z,
                            float4* xhi, float4* xlo, bool mixed, cudaStream_t stream)
{
    if (natoms <= 0) return;
    launch_pdl(k_split_positions, dim3((natoms + 255) / 256), dim3(256), 0, stream, pos, natoms, x, y, z, xhi, xlo, mixed);
}

void launch_coordination_number(const Batch& b, const Species& s, const Config& c,
                                const Partition& p, const Work& w, cudaStream_t stream, const InputPositions* in,
                                void* uv)
{
    if (b.natoms <= 0) return;
    if (!in && b.tiles && b.nid <= kMaxSpeciesFast) {
        launch_coordination_number_tiled(b, s, c, p, w, stream);
        return;
    }
    // small systems in input order: kDirectWarps warps per atom
    const dim3 grid(in ? blocks_for_atoms(b.natoms, kDirectWarps) : blocks_for_atoms(b.natoms)), block(kThreads);
    const InputPositions none{};
    if (c.mixed) {
        if (in)
            launch_pdl(k_coordination_number<float, true, kDirectWarps>, grid, block, 0, stream, b, s, c, p, w,
                       (float*)uv, *in);
        else
            launch_pdl(k_coordination_number<float, false, 1>, grid, block, 0, stream, b, s, c, p, w, (float*)nullptr,
                       none);
    } else {
        if (in)
            launch_pdl(k_coordination_number<double, true, kDirectWarps>, grid, block, 0, stream, b, s, c, p, w,
                       (double*)uv, *in);
        else
            launch_pdl(k_coordination_number<double, false, 1>, grid, block, 0, stream, b, s, c, p, w,
                       (double*)nullptr, none);
    }
}

void launch_weights(const Batch& b, const Species& s, const Config& c, const Work& w, cudaStream_t stream)
{
    if (b.natoms <= 0) return;
    launch_pdl(k_weights, dim3((b.natoms + 127) / 128), dim3(128), 0, stream, b, s, c, w);
}

void launch_two_body(const Batch& b, const Species& s, const Damp& d, const Config& c,
                     const Partition& p, const Work& w, cudaStream_t stream, const void* uv)
{
    if (b.natoms <= 0) return;
    if (!uv && b.tiles && b.nid <= kMaxSpeciesFast) {
        launch_two_body_tiled(b, s, d, c, p, w, stream);
        return;
    }
    const float* uf = (const float*)uv;
    const double* ud = (const double*)uv;
    // with the species vectors (small systems in input order): kDirectWarps warps per atom
#define D3_TB(R, DAMP, G, U)                                                                                  \
    launch_pdl(k_two_body<R, DAMP, G>, dim3(blocks_for_atoms(b.natoms, G)), dim3(kThreads), 0, stream, b, s, d, c, p, \
               w, U)
    if (d.kind == kRational) {
        if (c.mixed) { if (uv) D3_TB(float, kRational, kDirectWarps, uf); else D3_TB(float, kRational, 1, uf); }
        else { if (uv) D3_TB(double, kRational, kDirectWarps, ud); else D3_TB(double, kRational, 1, ud); }
    } else {
        if (c.mixed) { if (uv) D3_TB(float, kZero, kDirectWarps, uf); else D3_TB(float, kZero, 1, uf); }
        else { if (uv) D3_TB(double, kZero, kDirectWarps, ud); else D3_TB(double, kZero, 1, ud); }
    }
#undef D3_TB
}

void launch_cn_chain_rule(const Batch& b, const Species& s, const Config& c, const Partition& p,
                          const Work& w, cudaStream_t stream, bool direct)
{
    if (b.natoms <= 0) return;
    if (!direct && b.tiles && b.nid <= kMaxSpeciesFast) {
        launch_cn_chain_rule_tiled(b, s, c, p, w, stream);
        return;
    }
    const dim3 block(kThreads);
    if (direct) {
        const dim3 grid(blocks_for_atoms(b.natoms, kDirectWarps));
        if (c.mixed) launch_pdl(k_cn_chain<float, kDirectWarps>, grid, block, 0, stream, b, s, c, p, w);
        else launch_pdl(k_cn_chain<double, kDirectWarps>, grid, block, 0, stream, b, s, c, p, w);
    } else {
        const dim3 grid(blocks_for_atoms(b.natoms));
        if (c.mixed) launch_pdl(k_cn_chain<float, 1>, grid, block, 0, stream, b, s, c, p, w);
        else launch_pdl(k_cn_chain<double, 1>, grid, block, 0, stream, b, s, c, p, w);
    }
}

void launch_reduce_systems(const Batch& b, const Config& c, const Work& w, double* energies,
                           double* sigma9, double* param_grad, double* grad_out, cudaStream_t stream)
{
    if (b.nsys <= 0) return;
    // a block of 1024 threads where systems average above 512 atoms
    if (b.natoms > 512LL * b.nsys)
        launch_pdl(k_reduce_systems<1024>, dim3(b.nsys), dim3(1024), 0, stream, b, c, w, energies, sigma9, param_grad, grad_out);
    else
        launch_pdl(k_reduce_systems<256>, dim3(b.nsys), dim3(256), 0, stream, b, c, w, energies, sigma9, param_grad, grad_out);
}

}  // namespace d3
