// Analytic Hessian of the dispersion energy (get_dispersion_hessian,
// disp.f90:236-308), in FP64, for one structure in input atom order.  The
// kernels follow the reference's loops pair by pair (and triple by triple),
// so the work partition splits them as the reference does:
//
//   k_hs_cn       CN and B = dCN/dR [3N][N]   (counting function, ncoord.f90)
//   k_hs_weights  reference weights and their first two CN derivatives
//                 (model.f90:201-273)
//   k_hs_c6       C6, dC6/dCN and the second derivatives (model.f90:363-401)
//   k_hs_pair     two-body blocks, dE/dCN, A = d2E/dR dCN [3N][N] and
//                 D = d2E/dCN2 [N][N] from the family's damping kernel
//                 (damping.f90:393-539)
//   k_hs_triple   the same for the ATM term (atm.f90:38-429)
//   k_hs_cn_hess  the CN second derivative weighted by dE/dCN (ncoord.f90:230-306)
//   k_hs_xyt      C += X Y^T, for H += A B^T + B A^T + B D B^T (disp.f90:299-301)
//
// Blocks shared by several pairs or triples are added with FP64 atomics, so
// the last bits depend on the order of the additions.  This is an analysis
// path: O(N^2) memory and the plain loops of the reference.
#include <cfloat>
#include <cstdint>

#include "d3_device.cuh"

namespace d3 {

namespace {

constexpr int kHsThreads = 128;
constexpr double kKcnH = 16.0;        // ncoord.f90:31
constexpr double kWfH = 4.0;          // model.f90:80

struct HsSys {
    int n = 0, nid = 0;
    const double* pos = nullptr;      // [n][3] input order
    const int* sp = nullptr;          // [n] species
    const int* zid = nullptr;         // [n] species index inside the structure, from 1
    const uint8_t* ghost = nullptr;   // [n] or null
    const double* img = nullptr;      // lattice translations
    int img_cn0 = 0, img_cn1 = 0, img2_0 = 0, img2_1 = 0, img3_0 = 0, img3_1 = 0;
};

__device__ __forceinline__ bool hs_owns(const Partition& p, int i, int j)
{
    // partition.f90:127-147 on input indices
    if (p.nparts <= 1) return true;
    long long hi = i > j ? i : j, lo = i > j ? j : i;
    return (hi * (hi + 1) / 2 + lo) % p.nparts == p.part;
}

// pair (i, j <= i) of thread t in a lower-triangle sweep of n atoms; false
// beyond the triangle
__device__ __forceinline__ bool hs_pair(long long t, int n, int& i, int& j)
{
    i = (int)(t / n);
    j = (int)(t % n);
    return i < n && j <= i;
}

__global__ void k_hs_cn(HsSys h, Species s, double cutoff, double* cn, double* B)
{
    int i, j;
    if (!hs_pair(blockIdx.x * (long long)blockDim.x + threadIdx.x, h.n, i, j)) return;
    const int n = h.n;
    const double rc = s.rcov[h.sp[i]] + s.rcov[h.sp[j]];
    const double cut2 = cutoff * cutoff;
    double c = 0.0, g[3] = {0.0, 0.0, 0.0};
    for (int t = h.img_cn0; t < h.img_cn1; t++) {
        double v[3];
        for (int k = 0; k < 3; k++) v[k] = h.pos[3 * i + k] - (h.pos[3 * j + k] + h.img[3 * t + k]);
        const double r2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
        if (r2 > cut2 || r2 < 1.0e-12) continue;
        const double r1 = sqrt(r2);
        const double cf = 1.0 / (1.0 + exp(-kKcnH * (rc / r1 - 1.0)));
        c += cf;
        if (i == j) continue;
        const double dcf = -cf * (1.0 - cf) * kKcnH * rc / r2;
        for (int k = 0; k < 3; k++) g[k] += dcf * v[k] / r1;
    }
    if (c != 0.0) {
        atomicAdd(cn + i, c);
        if (i != j) atomicAdd(cn + j, c);
    }
    if (i == j) return;
    for (int k = 0; k < 3; k++) {
        if (g[k] == 0.0) continue;
        atomicAdd(B + (size_t)(3 * i + k) * n + i, g[k]);
        atomicAdd(B + (size_t)(3 * i + k) * n + j, g[k]);
        atomicAdd(B + (size_t)(3 * j + k) * n + i, -g[k]);
        atomicAdd(B + (size_t)(3 * j + k) * n + j, -g[k]);
    }
}

__global__ void k_hs_weights(HsSys h, Species s, const double* cn, double* gw, double* dgw, double* d2gw)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= h.n) return;
    const int sp = h.sp[i];
    const int nref = s.nref[sp];
    const double* cnref = s.refcn + sp * kMaxRef;
    const double wf2 = 2.0 * kWfH;
    double gwt[kMaxRef];
    double norm = 0.0, dnorm = 0.0, d2norm = 0.0, maxcn = cnref[0];
    for (int r = 0; r < nref; r++) {
        const double d = cn[i] - cnref[r];
        const double e = exp(-kWfH * d * d);
        gwt[r] = e;
        const double dcn = cnref[r] - cn[i];
        norm += e;
        dnorm += wf2 * dcn * e;
        d2norm += (wf2 * wf2 * dcn * dcn - wf2) * e;
        maxcn = fmax(maxcn, cnref[r]);
    }
    norm = 1.0 / norm;
    for (int r = 0; r < kMaxRef; r++) {
        double g0 = 0.0, g1 = 0.0, g2 = 0.0;
        if (r < nref) {
            const double expw = gwt[r], dcn = cnref[r] - cn[i];
            const double expd = wf2 * dcn * expw, expdd = (wf2 * wf2 * dcn * dcn - wf2) * expw;
            g0 = expw * norm;
            if (isnan(g0) || isinf(g0)) g0 = maxcn == cnref[r] ? 1.0 : 0.0;
            g1 = expd * norm - expw * dnorm * norm * norm;
            if (isnan(g1) || isinf(g1)) g1 = 0.0;
            g2 = expdd * norm - 2.0 * expd * dnorm * norm * norm - expw * d2norm * norm * norm
               + 2.0 * expw * dnorm * dnorm * norm * norm * norm;
            if (isnan(g2) || isinf(g2)) g2 = 0.0;
        }
        gw[i * kMaxRef + r] = g0;
        dgw[i * kMaxRef + r] = g1;
        d2gw[i * kMaxRef + r] = g2;
    }
}

// element (i, j) of each matrix at [i*n + j]: c6, dC6/dCN_i, d2C6/dCN_i^2 and
// the mixed d2C6/dCN_i dCN_j
__global__ void k_hs_c6(HsSys h, Species s, const double* gw, const double* dgw, const double* d2gw, double* c6,
                        double* dc6, double* d2c6, double* d2mix)
{
    int i, j;
    if (!hs_pair(blockIdx.x * (long long)blockDim.x + threadIdx.x, h.n, i, j)) return;
    const int n = h.n;
    double v = 0, di = 0, dj = 0, d2i = 0, d2j = 0, dm = 0;
    if (!(h.ghost && (h.ghost[i] || h.ghost[j]))) {
        const int si = h.sp[i], sj = h.sp[j];
        const double* ref = s.c6ref + (size_t)(si * h.nid + sj) * kMaxRef * kMaxRef;
        for (int ir = 0; ir < s.nref[si]; ir++)
            for (int jr = 0; jr < s.nref[sj]; jr++) {
                const double rc6 = ref[ir * kMaxRef + jr];
                const double gi = gw[i * kMaxRef + ir], gj = gw[j * kMaxRef + jr];
                const double dgi = dgw[i * kMaxRef + ir], dgj = dgw[j * kMaxRef + jr];
                v += gi * gj * rc6;
                di += dgi * gj * rc6;
                dj += gi * dgj * rc6;
                d2i += d2gw[i * kMaxRef + ir] * gj * rc6;
                d2j += gi * d2gw[j * kMaxRef + jr] * rc6;
                dm += dgi * dgj * rc6;
            }
    }
    c6[(size_t)i * n + j] = v; c6[(size_t)j * n + i] = v;
    dc6[(size_t)i * n + j] = di; dc6[(size_t)j * n + i] = dj;
    d2c6[(size_t)i * n + j] = d2i; d2c6[(size_t)j * n + i] = d2j;
    d2mix[(size_t)i * n + j] = dm; d2mix[(size_t)j * n + i] = dm;
}

__device__ void hs_smooth_r2(double r2, double cutoff, double width, double& sw, double& dsw, double& d2sw)
{
    // cutoff.f90:104-134
    const double r1 = sqrt(r2);
    double dswdr = 0.0, d2swdr2 = 0.0;
    sw = 1.0;
    if (width > 0.0 && width < cutoff) {
        if (r1 >= cutoff) {
            sw = 0.0;
        } else if (r1 > cutoff - width) {
            const double x = (cutoff - r1) / width;
            sw = x * x * x * (10.0 + x * (-15.0 + 6.0 * x));
            dswdr = -30.0 * x * x * (1.0 - x) * (1.0 - x) / width;
            d2swdr2 = 60.0 * x * (1.0 - x) * (1.0 - 2.0 * x) / (width * width);
        }
    }
    dsw = 0.5 * dswdr / r1;
    d2sw = 0.25 * (d2swdr2 - dswdr / r1) / r2;
}

// The family's pair kernel (get_damping_kernel of rational, zero, mzero,
// optimizedpower, cso and z.f90): e = -C6 p(u), u = r^2, and e_u, e_c,
// e_uu, e_uc, e_cc.
__device__ void hs_damping_kernel(const Damp& d, double rrij, double rvdw, int zsum, double u, double c6,
                                  double k[6])
{
    for (int q = 0; q < 6; q++) k[q] = 0.0;
    if (d.kind != kCSO && fabs(d.s6) < DBL_EPSILON && fabs(d.s8) < DBL_EPSILON) return;
    double pv, pd, pdd, pc = 0.0, puc = 0.0, pcc = 0.0;
    if (d.kind == kRational) {
        const double r0 = d.a1 * sqrt(rrij) + d.a2, r02 = r0 * r0, r06 = r02 * r02 * r02, r08 = r06 * r02;
        const double t6 = 1.0 / (u * u * u + r06), t8 = 1.0 / (u * u * u * u + r08);
        const double t6d = -3.0 * u * u * t6 * t6, t8d = -4.0 * u * u * u * t8 * t8;
        const double t6dd = -6.0 * u * t6 * t6 + 18.0 * pow(u, 4) * pow(t6, 3);
        const double t8dd = -12.0 * u * u * t8 * t8 + 32.0 * pow(u, 6) * pow(t8, 3);
        pv = d.s6 * t6 + d.s8 * rrij * t8;
        pd = d.s6 * t6d + d.s8 * rrij * t8d;
        pdd = d.s6 * t6dd + d.s8 * rrij * t8dd;
    } else if (d.kind == kZero || d.kind == kMZero) {
        const double alp6 = d.alp, alp8 = d.alp + 2.0;
        double t6, t8, t6d, t8d, t6dd, t8dd;
        if (d.kind == kZero) {
            const double a6 = 0.5 * alp6, a8 = 0.5 * alp8;
            t6 = pow(d.rs6 * rvdw / sqrt(u), alp6);
            t8 = pow(d.rs8 * rvdw / sqrt(u), alp8);
            t6d = -a6 * t6 / u;
            t8d = -a8 * t8 / u;
            t6dd = a6 * (a6 + 1.0) * t6 / (u * u);
            t8dd = a8 * (a8 + 1.0) * t8 / (u * u);
        } else {
            const double r1 = sqrt(u), betr0 = d.bet * rvdw;
            const double w6 = r1 / (d.rs6 * rvdw) + betr0, w8 = r1 / (d.rs8 * rvdw) + betr0;
            const double w6d = 1.0 / (d.rs6 * rvdw * 2.0 * r1), w8d = 1.0 / (d.rs8 * rvdw * 2.0 * r1);
            const double w6dd = -1.0 / (d.rs6 * rvdw * 4.0 * u * r1), w8dd = -1.0 / (d.rs8 * rvdw * 4.0 * u * r1);
            t6 = pow(w6, -alp6);
            t8 = pow(w8, -alp8);
            t6d = -alp6 * pow(w6, -alp6 - 1.0) * w6d;
            t8d = -alp8 * pow(w8, -alp8 - 1.0) * w8d;
            t6dd = alp6 * (alp6 + 1.0) * pow(w6, -alp6 - 2.0) * w6d * w6d - alp6 * pow(w6, -alp6 - 1.0) * w6dd;
            t8dd = alp8 * (alp8 + 1.0) * pow(w8, -alp8 - 2.0) * w8d * w8d - alp8 * pow(w8, -alp8 - 1.0) * w8dd;
        }
        const double f6 = 1.0 / (1.0 + 6.0 * t6), f8 = 1.0 / (1.0 + 6.0 * t8);
        const double f6d = -6.0 * t6d * f6 * f6, f8d = -6.0 * t8d * f8 * f8;
        const double f6dd = -6.0 * t6dd * f6 * f6 + 72.0 * t6d * t6d * pow(f6, 3);
        const double f8dd = -6.0 * t8dd * f8 * f8 + 72.0 * t8d * t8d * pow(f8, 3);
        const double c6t = f6 / pow(u, 3), c6td = f6d / pow(u, 3) - 3.0 * f6 / pow(u, 4);
        const double c6tdd = f6dd / pow(u, 3) - 6.0 * f6d / pow(u, 4) + 12.0 * f6 / pow(u, 5);
        const double c8t = f8 / pow(u, 4), c8td = f8d / pow(u, 4) - 4.0 * f8 / pow(u, 5);
        const double c8tdd = f8dd / pow(u, 4) - 8.0 * f8d / pow(u, 5) + 20.0 * f8 / pow(u, 6);
        pv = d.s6 * c6t + d.s8 * rrij * c8t;
        pd = d.s6 * c6td + d.s8 * rrij * c8td;
        pdd = d.s6 * c6tdd + d.s8 * rrij * c8tdd;
    } else if (d.kind == kOptimizedPower) {
        const double r0 = d.a1 * sqrt(rrij) + d.a2, r02 = r0 * r0, r06 = r02 * r02 * r02, r08 = r06 * r02;
        const double ab = pow(r0, d.bet), a6 = ab * r06, a8 = ab * r08, q = 0.5 * d.bet;
        const double d6 = pow(u, 3) + a6 * pow(u, -q), d8 = pow(u, 4) + a8 * pow(u, -q);
        const double d6d = 3.0 * u * u - q * a6 * pow(u, -q - 1.0), d8d = 4.0 * pow(u, 3) - q * a8 * pow(u, -q - 1.0);
        const double d6dd = 6.0 * u + q * (q + 1.0) * a6 * pow(u, -q - 2.0);
        const double d8dd = 12.0 * u * u + q * (q + 1.0) * a8 * pow(u, -q - 2.0);
        const double t6 = 1.0 / d6, t8 = 1.0 / d8;
        const double t6d = -d6d * t6 * t6, t8d = -d8d * t8 * t8;
        const double t6dd = -d6dd * t6 * t6 + 2.0 * d6d * d6d * pow(t6, 3);
        const double t8dd = -d8dd * t8 * t8 + 2.0 * d8d * d8d * pow(t8, 3);
        pv = d.s6 * t6 + d.s8 * rrij * t8;
        pd = d.s6 * t6d + d.s8 * rrij * t8d;
        pdd = d.s6 * t6dd + d.s8 * rrij * t8dd;
    } else if (d.kind == kCSO) {
        const double r1 = sqrt(u), r0 = sqrt(rrij);
        const double dd6_6 = pow(d.rs6 * r0 + d.rs8, 6);
        const double sf = 1.0 / (1.0 + exp(r1 - d.a2 * r0));
        const double sfd = -sf * (1.0 - sf), sfdd = sf * (1.0 - sf) * (1.0 - 2.0 * sf);
        const double sig = d.s6 + d.a1 * sf, sigd = d.a1 * sfd, sigdd = d.a1 * sfdd;
        const double sigu = 0.5 * sigd / r1, siguu = 0.25 * sigdd / u - 0.25 * sigd / (u * r1);
        const double t6 = 1.0 / (u * u * u + dd6_6);
        const double t6d = -3.0 * u * u * t6 * t6, t6dd = -6.0 * u * t6 * t6 + 18.0 * pow(u, 4) * pow(t6, 3);
        pv = sig * t6;
        pd = sigu * t6 + sig * t6d;
        pdd = siguu * t6 + 2.0 * sigu * t6d + sig * t6dd;
    } else {
        const double r0 = d.a1 / double(zsum), b8 = r0 * rrij;
        const double t6 = 1.0 / (u * u * u + r0 * c6), t8 = 1.0 / (u * u * u * u + b8 * c6);
        const double t6u = -3.0 * u * u * t6 * t6, t8u = -4.0 * pow(u, 3) * t8 * t8;
        const double t6uu = -6.0 * u * t6 * t6 + 18.0 * pow(u, 4) * pow(t6, 3);
        const double t8uu = -12.0 * u * u * t8 * t8 + 32.0 * pow(u, 6) * pow(t8, 3);
        const double t6c = -r0 * t6 * t6, t8c = -b8 * t8 * t8;
        const double t6uc = 6.0 * u * u * r0 * pow(t6, 3), t8uc = 8.0 * pow(u, 3) * b8 * pow(t8, 3);
        const double t6cc = 2.0 * r0 * r0 * pow(t6, 3), t8cc = 2.0 * b8 * b8 * pow(t8, 3);
        pv = d.s6 * t6 + d.s8 * rrij * t8;
        pd = d.s6 * t6u + d.s8 * rrij * t8u;
        pdd = d.s6 * t6uu + d.s8 * rrij * t8uu;
        pc = d.s6 * t6c + d.s8 * rrij * t8c;
        puc = d.s6 * t6uc + d.s8 * rrij * t8uc;
        pcc = d.s6 * t6cc + d.s8 * rrij * t8cc;
    }
    k[0] = -c6 * pv;
    k[1] = -c6 * pd;
    k[2] = -pv - c6 * pc;
    k[3] = -c6 * pdd;
    k[4] = -pd - c6 * puc;
    k[5] = -2.0 * pc - c6 * pcc;
}

struct HsMats {
    const double *c6, *dc6, *d2c6, *d2mix;   // [n][n]
    double *H;                               // [3n][3n]
    double *dEdcn;                           // [n]
    double *A;                               // [3n][n]
    double *D;                               // [n][n]
};

__global__ void k_hs_pair(HsSys h, Species s, Damp d, Config c, Partition part, const double* rvdw, HsMats m)
{
    int i, j;
    if (!hs_pair(blockIdx.x * (long long)blockDim.x + threadIdx.x, h.n, i, j)) return;
    if (!hs_owns(part, i, j)) return;
    const int n = h.n;
    const size_t n3 = 3 * (size_t)n;
    const int si = h.sp[i], sj = h.sp[j];
    const double rrij = s.pair[kPairSlots * (si * h.nid + sj)];
    const double r0 = rvdw[sj * h.nid + si];
    const int zsum = h.zid[i] + h.zid[j];
    const double c6ij = m.c6[(size_t)j * n + i];
    double fac;
    int nc, cnat[2];
    double cnd[2], cnd2[2][2];
    if (i != j) {
        fac = 1.0; nc = 2; cnat[0] = i; cnat[1] = j;
        cnd[0] = m.dc6[(size_t)i * n + j];
        cnd[1] = m.dc6[(size_t)j * n + i];
        cnd2[0][0] = m.d2c6[(size_t)i * n + j];
        cnd2[1][1] = m.d2c6[(size_t)j * n + i];
        cnd2[0][1] = cnd2[1][0] = m.d2mix[(size_t)i * n + j];
    } else {
        fac = 0.5; nc = 1; cnat[0] = i; cnat[1] = i;
        cnd[0] = 2.0 * m.dc6[(size_t)i * n + i];
        cnd[1] = 0.0;
        cnd2[0][0] = 2.0 * m.d2c6[(size_t)i * n + i] + 2.0 * m.d2mix[(size_t)i * n + i];
        cnd2[0][1] = cnd2[1][0] = cnd2[1][1] = 0.0;
    }
    const double cut2 = c.cut2 * c.cut2;
    // sums over the translations: geometric block, dE/dCN, D and A terms
    double blk[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    double sfc = 0.0, sfcc = 0.0, avec[3] = {0, 0, 0};
    for (int t = h.img2_0; t < h.img2_1; t++) {
        double v[3];
        for (int k = 0; k < 3; k++) v[k] = h.pos[3 * i + k] - (h.pos[3 * j + k] + h.img[3 * t + k]);
        const double r2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
        if (r2 > cut2 || r2 < DBL_EPSILON) continue;
        double k6[6], sw, swr, swrr;
        hs_damping_kernel(d, rrij, r0, zsum, r2, c6ij, k6);
        hs_smooth_r2(r2, c.cut2, c.width2, sw, swr, swrr);
        const double fr = fac * (swr * k6[0] + sw * k6[1]);
        const double frr = fac * (swrr * k6[0] + 2.0 * swr * k6[1] + sw * k6[3]);
        const double fc = fac * sw * k6[2];
        const double frc = fac * (swr * k6[2] + sw * k6[4]);
        const double fcc = fac * sw * k6[5];
        if (i != j) {
            for (int a = 0; a < 3; a++) {
                for (int b = 0; b < 3; b++) blk[a][b] += 4.0 * frr * v[a] * v[b];
                blk[a][a] += 2.0 * fr;
                avec[a] += frc * 2.0 * v[a];
            }
        }
        sfc += fc;
        sfcc += fcc;
    }
    if (i != j) {
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) {
                const double x = blk[a][b];
                if (x == 0.0) continue;
                atomicAdd(m.H + (3 * i + a) * n3 + 3 * i + b, x);
                atomicAdd(m.H + (3 * j + a) * n3 + 3 * j + b, x);
                atomicAdd(m.H + (3 * i + a) * n3 + 3 * j + b, -x);
                atomicAdd(m.H + (3 * j + a) * n3 + 3 * i + b, -x);
            }
    }
    for (int ia = 0; ia < nc; ia++) {
        if (sfc != 0.0) atomicAdd(m.dEdcn + cnat[ia], sfc * cnd[ia]);
        for (int ib = 0; ib < nc; ib++) {
            const double x = sfcc * cnd[ia] * cnd[ib] + sfc * cnd2[ia][ib];
            if (x != 0.0) atomicAdd(m.D + (size_t)cnat[ia] * n + cnat[ib], x);
        }
    }
    if (i != j) {
        for (int ia = 0; ia < nc; ia++)
            for (int a = 0; a < 3; a++) {
                const double x = avec[a] * cnd[ia];
                if (x == 0.0) continue;
                atomicAdd(m.A + (size_t)(3 * i + a) * n + cnat[ia], x);
                atomicAdd(m.A + (size_t)(3 * j + a) * n + cnat[ia], -x);
            }
    }
}

__device__ __forceinline__ double hs_triple_scale(int i, int j, int k)
{
    // atm.f90:954-980
    if (i == j) return i == k ? 1.0 / 6.0 : 0.5;
    return (i != k && j != k) ? 1.0 : 0.5;
}

__global__ void __launch_bounds__(kHsThreads) k_hs_triple(HsSys h, Species s, Damp d, Config c, Partition part,
                                                          HsMats m)
{
    int i, j;
    if (!hs_pair(blockIdx.x * (long long)blockDim.x + threadIdx.x, h.n, i, j)) return;
    if (!hs_owns(part, i, j)) return;
    // [atom][pair] coefficients of the pair vectors x_j - x_i, x_k - x_i, x_k - x_j
    const int sigp[3][3] = {{-1, -1, 0}, {1, 0, -1}, {0, 1, 1}};
    // d l / d u: l1 = u1 - u2 + u3, l2 = u1 + u2 - u3, l3 = -u1 + u2 + u3
    const double cl[3][3] = {{1, -1, 1}, {1, 1, -1}, {-1, 1, 1}};
    const int n = h.n;
    const size_t n3 = 3 * (size_t)n;
    const double cut2 = c.cut3 * c.cut3;
    const double alp3 = (d.alp + 2.0) / 3.0, aexp = 0.5 * alp3;
    const int si = h.sp[i], sj = h.sp[j];
    for (int jt = h.img3_0; jt < h.img3_1; jt++) {
        double vec[3][3], u[3];
        for (int q = 0; q < 3; q++) vec[0][q] = h.pos[3 * j + q] + h.img[3 * jt + q] - h.pos[3 * i + q];
        u[0] = vec[0][0] * vec[0][0] + vec[0][1] * vec[0][1] + vec[0][2] * vec[0][2];
        if (u[0] > cut2 || u[0] < DBL_EPSILON) continue;
        for (int kk = 0; kk <= j; kk++) {
            const int sk = h.sp[kk];
            const double triple = hs_triple_scale(i, j, kk);
            const double r0 = s.atm_r0[sj * h.nid + si] * s.atm_r0[sk * h.nid + si] * s.atm_r0[sk * h.nid + sj];
            const double c6t[3] = {m.c6[(size_t)j * n + i], m.c6[(size_t)kk * n + i], m.c6[(size_t)kk * n + j]};
            if (fabs(c6t[0]) < DBL_EPSILON || fabs(c6t[1]) < DBL_EPSILON || fabs(c6t[2]) < DBL_EPSILON) continue;
            for (int kt = h.img3_0; kt < h.img3_1; kt++) {
                for (int q = 0; q < 3; q++) vec[1][q] = h.pos[3 * kk + q] + h.img[3 * kt + q] - h.pos[3 * i + q];
                u[1] = vec[1][0] * vec[1][0] + vec[1][1] * vec[1][1] + vec[1][2] * vec[1][2];
                if (u[1] > cut2 || u[1] < DBL_EPSILON) continue;
                for (int q = 0; q < 3; q++) vec[2][q] = vec[1][q] - vec[0][q];
                u[2] = vec[2][0] * vec[2][0] + vec[2][1] * vec[2][1] + vec[2][2] * vec[2][2];
                if (u[2] > cut2 || u[2] < DBL_EPSILON) continue;
                double swp[3], dswp[3], d2swp[3];
                for (int q = 0; q < 3; q++) hs_smooth_r2(u[q], c.cut3, c.width3, swp[q], dswp[q], d2swp[q]);
                const double sval = swp[0] * swp[1] * swp[2];
                const double sp[3] = {dswp[0] * swp[1] * swp[2], swp[0] * dswp[1] * swp[2], swp[0] * swp[1] * dswp[2]};
                double spq[3][3];
                spq[0][0] = d2swp[0] * swp[1] * swp[2];
                spq[1][1] = swp[0] * d2swp[1] * swp[2];
                spq[2][2] = swp[0] * swp[1] * d2swp[2];
                spq[0][1] = spq[1][0] = dswp[0] * dswp[1] * swp[2];
                spq[0][2] = spq[2][0] = dswp[0] * swp[1] * dswp[2];
                spq[1][2] = spq[2][1] = swp[0] * dswp[1] * dswp[2];
                const double ww = u[0] * u[1] * u[2];
                const double wp[3] = {u[1] * u[2], u[0] * u[2], u[0] * u[1]};
                const double wpq[3][3] = {{0, u[2], u[1]}, {u[2], 0, u[0]}, {u[1], u[0], 0}};
                const double lval[3] = {u[0] + u[2] - u[1], u[0] - u[2] + u[1], -u[0] + u[2] + u[1]};
                const double nval = lval[0] * lval[1] * lval[2];
                double np[3], npq[3][3];
                for (int a = 0; a < 3; a++)
                    np[a] = cl[0][a] * lval[1] * lval[2] + cl[1][a] * lval[0] * lval[2] + cl[2][a] * lval[0] * lval[1];
                for (int a = 0; a < 3; a++)
                    for (int b = 0; b < 3; b++) {
                        double tmp = 0.0;
                        for (int il = 0; il < 3; il++)
                            for (int im = 0; im < 3; im++)
                                if (il != im) tmp += cl[il][a] * cl[im][b] * lval[3 - il - im];
                        npq[a][b] = tmp;
                    }
                const double gv = pow(ww, -2.5), gd = -2.5 * pow(ww, -3.5), gdd = 8.75 * pow(ww, -4.5);
                const double hv = pow(ww, -1.5), hd = -1.5 * pow(ww, -2.5), hdd = 3.75 * pow(ww, -3.5);
                const double ang = 0.375 * nval * gv + hv;
                double angp[3], angpq[3][3];
                for (int a = 0; a < 3; a++) angp[a] = 0.375 * (np[a] * gv + nval * gd * wp[a]) + hd * wp[a];
                for (int a = 0; a < 3; a++)
                    for (int b = 0; b < 3; b++)
                        angpq[a][b] = 0.375 * (npq[a][b] * gv + np[a] * gd * wp[b] + np[b] * gd * wp[a]
                                               + nval * (gdd * wp[a] * wp[b] + gd * wpq[a][b]))
                                    + hdd * wp[a] * wp[b] + hd * wpq[a][b];
                const double tval = 6.0 * pow(r0, alp3) * pow(ww, -aexp);
                double tp[3], tpq[3][3];
                for (int a = 0; a < 3; a++) tp[a] = -aexp * tval * wp[a] / ww;
                for (int a = 0; a < 3; a++)
                    for (int b = 0; b < 3; b++)
                        tpq[a][b] = aexp * (aexp + 1.0) * tval * wp[a] * wp[b] / (ww * ww) - aexp * tval * wpq[a][b] / ww;
                const double fd = 1.0 / (1.0 + tval);
                double fdp[3], fdpq[3][3];
                for (int a = 0; a < 3; a++) fdp[a] = -tp[a] * fd * fd;
                for (int a = 0; a < 3; a++)
                    for (int b = 0; b < 3; b++) fdpq[a][b] = -tpq[a][b] * fd * fd + 2.0 * tp[a] * tp[b] * fd * fd * fd;
                const double av = ang * fd;
                double ap[3], kp[3], kpq[3][3];
                for (int a = 0; a < 3; a++) ap[a] = angp[a] * fd + ang * fdp[a];
                const double kv = sval * av;
                for (int a = 0; a < 3; a++) kp[a] = sp[a] * av + sval * ap[a];
                for (int a = 0; a < 3; a++)
                    for (int b = 0; b < 3; b++) {
                        const double apq = angpq[a][b] * fd + angp[a] * fdp[b] + angp[b] * fdp[a] + ang * fdpq[a][b];
                        kpq[a][b] = spq[a][b] * av + sp[a] * ap[b] + sp[b] * ap[a] + sval * apq;
                    }
                const double qv = sqrt(fabs(c6t[0] * c6t[1] * c6t[2]));
                const double pref = d.s9 * triple, pq = pref * qv;
                const int at[3] = {i, j, kk};
                // gradient of u_q with respect to atom a: 2 sigp[a][q] vec_q
                double gk[3][3][3];                  // [c][atom][pair]
                for (int a = 0; a < 3; a++)
                    for (int cc = 0; cc < 3; cc++)
                        for (int q = 0; q < 3; q++) {
                            double tmp = 0.0;
                            for (int sdx = 0; sdx < 3; sdx++) tmp += kpq[sdx][q] * 2.0 * sigp[a][sdx] * vec[sdx][cc];
                            gk[cc][a][q] = pq * tmp;
                        }
                for (int a = 0; a < 3; a++)
                    for (int b = 0; b < 3; b++) {
                        double dg = 0.0;
                        for (int sdx = 0; sdx < 3; sdx++) dg += kp[sdx] * sigp[a][sdx] * sigp[b][sdx];
                        dg *= 2.0 * pq;
                        for (int cc = 0; cc < 3; cc++)
                            for (int dd = 0; dd < 3; dd++) {
                                double tmp = cc == dd ? dg : 0.0;
                                for (int q = 0; q < 3; q++) tmp += gk[cc][a][q] * 2.0 * sigp[b][q] * vec[q][dd];
                                atomicAdd(m.H + (size_t)(3 * at[a] + cc) * n3 + 3 * at[b] + dd, tmp);
                            }
                    }
                double ec[3], ecc[3][3];
                for (int a = 0; a < 3; a++) {
                    ec[a] = pref * 0.5 * qv / c6t[a] * kv;
                    for (int b = 0; b < 3; b++)
                        ecc[a][b] = pref * kv * (a == b ? -0.25 * qv / (c6t[a] * c6t[a]) : 0.25 * qv / (c6t[a] * c6t[b]));
                }
                const int pat[3][2] = {{i, j}, {i, kk}, {j, kk}};
                int nent = 0, ent_atom[6], ent_pair[6];
                double ent_coef[6];
                for (int q = 0; q < 3; q++) {
                    const int a1 = pat[q][0], a2 = pat[q][1];
                    if (a1 != a2) {
                        ent_atom[nent] = a1; ent_pair[nent] = q; ent_coef[nent++] = m.dc6[(size_t)a1 * n + a2];
                        ent_atom[nent] = a2; ent_pair[nent] = q; ent_coef[nent++] = m.dc6[(size_t)a2 * n + a1];
                    } else {
                        ent_atom[nent] = a1; ent_pair[nent] = q; ent_coef[nent++] = 2.0 * m.dc6[(size_t)a1 * n + a1];
                    }
                }
                for (int e = 0; e < nent; e++) {
                    const int q = ent_pair[e];
                    atomicAdd(m.dEdcn + ent_atom[e], ec[q] * ent_coef[e]);
                    for (int f = 0; f < nent; f++)
                        atomicAdd(m.D + (size_t)ent_atom[e] * n + ent_atom[f], ecc[q][ent_pair[f]] * ent_coef[e] * ent_coef[f]);
                    // d2E/dR dCN: pref qm_q kp_s du_s/dR
                    const double eu = pref * 0.5 * qv / c6t[q];
                    for (int a = 0; a < 3; a++)
                        for (int cc = 0; cc < 3; cc++) {
                            double tmp = 0.0;
                            for (int sdx = 0; sdx < 3; sdx++) tmp += eu * kp[sdx] * 2.0 * sigp[a][sdx] * vec[sdx][cc];
                            atomicAdd(m.A + (size_t)(3 * at[a] + cc) * n + ent_atom[e], tmp * ent_coef[e]);
                        }
                }
                for (int q = 0; q < 3; q++) {
                    const int a1 = pat[q][0], a2 = pat[q][1];
                    if (a1 != a2) {
                        atomicAdd(m.D + (size_t)a1 * n + a1, ec[q] * m.d2c6[(size_t)a1 * n + a2]);
                        atomicAdd(m.D + (size_t)a2 * n + a2, ec[q] * m.d2c6[(size_t)a2 * n + a1]);
                        atomicAdd(m.D + (size_t)a1 * n + a2, ec[q] * m.d2mix[(size_t)a1 * n + a2]);
                        atomicAdd(m.D + (size_t)a2 * n + a1, ec[q] * m.d2mix[(size_t)a1 * n + a2]);
                    } else {
                        atomicAdd(m.D + (size_t)a1 * n + a1,
                                  ec[q] * (2.0 * m.d2c6[(size_t)a1 * n + a1] + 2.0 * m.d2mix[(size_t)a1 * n + a1]));
                    }
                }
            }
        }
    }
}

__global__ void k_hs_cn_hess(HsSys h, Species s, double cutoff, const double* dEdcn, double* H)
{
    int i, j;
    if (!hs_pair(blockIdx.x * (long long)blockDim.x + threadIdx.x, h.n, i, j) || j == i) return;
    const size_t n3 = 3 * (size_t)h.n;
    const double rc = s.rcov[h.sp[i]] + s.rcov[h.sp[j]];
    const double de = dEdcn[i] + dEdcn[j];
    const double cut2 = cutoff * cutoff;
    double blk[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (int t = h.img_cn0; t < h.img_cn1; t++) {
        double v[3];
        for (int k = 0; k < 3; k++) v[k] = h.pos[3 * i + k] - (h.pos[3 * j + k] + h.img[3 * t + k]);
        const double r2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
        if (r2 > cut2 || r2 < 1.0e-12) continue;
        const double r1 = sqrt(r2);
        const double cf = 1.0 / (1.0 + exp(-kKcnH * (rc / r1 - 1.0)));
        const double tmp = cf * (1.0 - cf);
        const double dcf = -tmp * kKcnH * rc / r2;
        const double d2cf = tmp * (1.0 - 2.0 * cf) * (kKcnH * rc) * (kKcnH * rc) / (r2 * r2)
                          + 2.0 * tmp * kKcnH * rc / (r2 * r1);
        for (int a = 0; a < 3; a++) {
            for (int b = 0; b < 3; b++) blk[a][b] += de * (d2cf * v[a] * v[b] / r2 - dcf * v[a] * v[b] / (r2 * r1));
            blk[a][a] += de * dcf / r1;
        }
    }
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) {
            const double x = blk[a][b];
            if (x == 0.0) continue;
            atomicAdd(H + (3 * i + a) * n3 + 3 * i + b, x);
            atomicAdd(H + (3 * j + a) * n3 + 3 * j + b, x);
            atomicAdd(H + (3 * i + a) * n3 + 3 * j + b, -x);
            atomicAdd(H + (3 * j + a) * n3 + 3 * i + b, -x);
        }
}

// C[r][q] += sum_k X[r][k] Y[q][k] for r < M, q < N, k < K (row-major, FP64),
// 16 x 16 tiles staged in shared memory
constexpr int kXyt = 16;
__global__ void k_hs_xyt(const double* X, const double* Y, double* C, int M, int N, int K, int ldc)
{
    __shared__ double xs[kXyt][kXyt + 1], ys[kXyt][kXyt + 1];
    const int r = blockIdx.y * kXyt + threadIdx.y, q = blockIdx.x * kXyt + threadIdx.x;
    double acc = 0.0;
    for (int k0 = 0; k0 < K; k0 += kXyt) {
        const int kx = k0 + threadIdx.x;
        const int ry = blockIdx.y * kXyt + threadIdx.y, qy = blockIdx.x * kXyt + threadIdx.y;
        xs[threadIdx.y][threadIdx.x] = (ry < M && kx < K) ? X[(size_t)ry * K + kx] : 0.0;
        ys[threadIdx.y][threadIdx.x] = (qy < N && kx < K) ? Y[(size_t)qy * K + kx] : 0.0;
        __syncthreads();
        for (int k = 0; k < kXyt; k++) acc += xs[threadIdx.y][k] * ys[threadIdx.x][k];
        __syncthreads();
    }
    if (r < M && q < N) C[(size_t)r * ldc + q] += acc;
}

void launch_xyt(const double* X, const double* Y, double* C, int M, int N, int K, cudaStream_t stream)
{
    const dim3 block(kXyt, kXyt), grid((N + kXyt - 1) / kXyt, (M + kXyt - 1) / kXyt);
    k_hs_xyt<<<grid, block, 0, stream>>>(X, Y, C, M, N, K, N);
}

}  // namespace

size_t hessian_scratch_doubles(int n)
{
    // cn, weights (3 x 7 n), four C6 matrices, dE/dCN, B, A, D, D B^T
    const size_t nn = (size_t)n * n;
    return (size_t)n + 3 * (size_t)kMaxRef * n + 4 * nn + (size_t)n + 3 * nn + 3 * nn + nn + 3 * nn;
}

void launch_hessian(const Species& s, const Damp& d, const Config& c, const Partition& p, int n, int nid,
                    const double* pos, const int* sp, const int* zid, const uint8_t* ghost, const double* img,
                    const int img_range[6], const double* rvdw, double* scratch, double* H, cudaStream_t stream)
{
    if (n <= 0) return;
    HsSys h;
    h.n = n; h.nid = nid; h.pos = pos; h.sp = sp; h.zid = zid; h.ghost = ghost; h.img = img;
    h.img_cn0 = img_range[0]; h.img_cn1 = img_range[1];
    h.img2_0 = img_range[2]; h.img2_1 = img_range[3];
    h.img3_0 = img_range[4]; h.img3_1 = img_range[5];
    const size_t nn = (size_t)n * n;
    double* cn = scratch;
    double* gw = cn + n;
    double* dgw = gw + (size_t)kMaxRef * n;
    double* d2gw = dgw + (size_t)kMaxRef * n;
    double* c6 = d2gw + (size_t)kMaxRef * n;
    double* dc6 = c6 + nn;
    double* d2c6 = dc6 + nn;
    double* d2mix = d2c6 + nn;
    double* dEdcn = d2mix + nn;
    double* B = dEdcn + n;
    double* A = B + 3 * nn;
    double* D = A + 3 * nn;
    double* DB = D + nn;
    cudaMemsetAsync(scratch, 0, sizeof(double) * hessian_scratch_doubles(n), stream);
    cudaMemsetAsync(H, 0, sizeof(double) * 9 * nn, stream);
    const unsigned pblocks = (unsigned)((nn + kHsThreads - 1) / kHsThreads);
    k_hs_cn<<<pblocks, kHsThreads, 0, stream>>>(h, s, c.cut_cn, cn, B);
    k_hs_weights<<<(n + kHsThreads - 1) / kHsThreads, kHsThreads, 0, stream>>>(h, s, cn, gw, dgw, d2gw);
    k_hs_c6<<<pblocks, kHsThreads, 0, stream>>>(h, s, gw, dgw, d2gw, c6, dc6, d2c6, d2mix);
    HsMats m{c6, dc6, d2c6, d2mix, H, dEdcn, A, D};
    k_hs_pair<<<pblocks, kHsThreads, 0, stream>>>(h, s, d, c, p, rvdw, m);
    if (std::fabs(d.s9) >= DBL_EPSILON) k_hs_triple<<<pblocks, kHsThreads, 0, stream>>>(h, s, d, c, p, m);
    k_hs_cn_hess<<<pblocks, kHsThreads, 0, stream>>>(h, s, c.cut_cn, dEdcn, H);
    // H += A B^T + B A^T + B (D B^T); DB[b][k] = sum_l B[b][l] D[k][l]
    const int n3 = 3 * n;
    launch_xyt(A, B, H, n3, n3, n, stream);
    launch_xyt(B, A, H, n3, n3, n, stream);
    launch_xyt(B, D, DB, n3, n, n, stream);
    launch_xyt(B, DB, H, n3, n3, n, stream);
}

}  // namespace d3
