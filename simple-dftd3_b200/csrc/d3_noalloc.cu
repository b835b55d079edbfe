// Allocation-free entry point: the two-body dispersion pipeline (coordination
// numbers, reference weights, two-body sum, CN chain rule, reduction) of one
// system with all device work arrays carved out of a fixed, file-scope
// __device__ array instead of cudaMalloc'd workspace.
//
// Who needs it: callers that must not allocate device memory at call time --
// integrators and MD engines that own every byte of device memory through
// their own pool allocator (a cudaMalloc behind the pool's back can fail or
// fragment the pool), and time-step loops in which cudaMalloc/cudaFree are
// not allowed because they can synchronise the whole device.  The caller
// passes device input and output buffers; the library allocates nothing, on
// the device or on the host heap (host-side tables live in fixed static
// buffers).
//
// Host blocking: the per-call tables are copied from those static host
// buffers on `stream`, and the call then waits for the stream
// (cudaStreamSynchronize) before the buffers can be reused, so it returns
// only after all work queued earlier on `stream` and its copies are done; the
// kernels themselves run asynchronously after it returns.
//
// Limits and sharing:
//   * at most kNoAllocMaxAtoms atoms, kNoAllocMaxSpecies distinct elements and
//     kNoAllocMaxImages lattice translations per cutoff; larger inputs are
//     rejected with an error before anything is launched;
//   * the scratch array (kNoAllocScratchBytes) belongs to the library: every
//     GPU that loads the library holds it until the process exits;
//   * every call on a device uses the same array and leaves the last call's
//     contents in it; calls whose work overlaps on the GPU (different streams,
//     or different host threads on one device) race on it and must be
//     serialised by the caller;
//   * the first call on a device resolves the device address of the array
//     (cudaGetSymbolAddress) with that device current; make this first call
//     before any stream capture.
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/dftd3_b200.h"
#include "d3_device.cuh"
#include "d3_engine.h"
#include "d3_tables.h"

namespace {

constexpr int kNoAllocMaxAtoms = 4096;
constexpr int kNoAllocMaxSpecies = 16;
constexpr int kNoAllocMaxImages = 8192;
constexpr size_t kNoAllocScratchBytes = size_t(4) << 20;   // 4 MiB
constexpr int kMaxDevices = 64;

// Device scratch shared by all calls on a device.  Host code must not use the
// name as an address: it is a host-side stand-in for the device symbol.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_mutex;                       // serialises the host-side staging below
unsigned char* g_scratch_ptr[kMaxDevices] = {};

// Host staging of the per-call tables (fixed size, no heap allocation).
struct HostStage {
    int atom_off[2];
    int img_off[d3::kImageKinds * 2];
    int nref[kNoAllocMaxSpecies];
    int num[kNoAllocMaxSpecies];
    int sp[kNoAllocMaxAtoms];
    int zeros[kNoAllocMaxAtoms];
    int local[kNoAllocMaxAtoms];
    double rcov[kNoAllocMaxSpecies];
    double r4r2[kNoAllocMaxSpecies];
    double rvdw[kNoAllocMaxSpecies * kNoAllocMaxSpecies];
    double refcn[kNoAllocMaxSpecies * d3::kMaxRef];
    double c6ref[kNoAllocMaxSpecies * kNoAllocMaxSpecies * d3::kMaxRef * d3::kMaxRef];
    float c6ref_f[kNoAllocMaxSpecies * kNoAllocMaxSpecies * d3::kMaxRef * d3::kMaxRef];
    double pair[kNoAllocMaxSpecies * kNoAllocMaxSpecies * d3::kPairSlots];
    double img[3 * kNoAllocMaxImages * d3::kImageKinds];
};
HostStage g_host;

// Bump allocator over the scratch array (256-byte aligned carve-outs).
struct Carver {
    unsigned char* base;
    size_t used = 0;
    bool overflow = false;
    template <class T>
    T* take(size_t n)
    {
        size_t off = (used + 255) & ~size_t(255);
        size_t bytes = n * sizeof(T);
        if (off + bytes > kNoAllocScratchBytes) {
            overflow = true;
            return nullptr;
        }
        used = off + bytes;
        return reinterpret_cast<T*>(base + off);
    }
};

// Lattice translations into a fixed buffer (get_lattice_points,
// cutoff.f90:140-227, same algorithm as d3::lattice_points); -1 if they do
// not fit.
int lattice_points_into(const double* lattice, const bool* periodic, double rthr, double* out, int cap)
{
    const int np = (int)periodic[0] + (int)periodic[1] + (int)periodic[2];
    if (np == 0) {
        if (cap < 1) return -1;
        out[0] = out[1] = out[2] = 0.0;
        return 1;
    }
    auto cross = [](const double* a, const double* b, double* c) {
        const double x = a[1] * b[2] - b[1] * a[2];
        const double y = a[2] * b[0] - b[2] * a[0];
        const double z = a[0] * b[1] - b[0] * a[1];
        c[0] = x; c[1] = y; c[2] = z;
    };
    // repetitions ceil(x) of one direction; -1 for a degenerate lattice (a zero
    // vector or normal gives x = inf or NaN) or more images than fit
    auto reps = [&](double x) {
        if (!(x >= 0.0) || x > (double)cap) return -1;
        return (int)std::ceil(x);
    };
    auto translations = [&](const double lat[3][3], int rep[3]) {
        double nrm[3][3];
        cross(lat[1], lat[2], nrm[0]);
        cross(lat[2], lat[0], nrm[1]);
        cross(lat[0], lat[1], nrm[2]);
        for (int k = 0; k < 3; k++) {
            const double n = std::sqrt(nrm[k][0] * nrm[k][0] + nrm[k][1] * nrm[k][1] + nrm[k][2] * nrm[k][2]);
            for (int c = 0; c < 3; c++) nrm[k][c] /= n;
        }
        for (int k = 0; k < 3; k++) {
            const double cs = nrm[k][0] * lat[k][0] + nrm[k][1] * lat[k][1] + nrm[k][2] * lat[k][2];
            rep[k] = reps(std::fabs(rthr / cs));
        }
    };
    double lat[3][3];
    for (int k = 0; k < 3; k++)
        for (int c = 0; c < 3; c++) lat[k][c] = lattice[3 * k + c];
    int rep[3] = {0, 0, 0};
    if (np == 3) {
        translations(lat, rep);
    } else if (np == 1) {
        for (int k = 0; k < 3; k++) {
            const double v = std::sqrt(lat[k][0] * lat[k][0] + lat[k][1] * lat[k][1] + lat[k][2] * lat[k][2]);
            rep[k] = periodic[k] ? reps(rthr / v) : 0;
        }
    } else {
        double nrm[3][3];
        for (int k = 0; k < 3; k++) cross(lat[(k + 1) % 3], lat[(k + 2) % 3], nrm[k]);
        for (int k = 0; k < 3; k++)
            for (int c = 0; c < 3; c++)
                if (periodic[c]) nrm[k][c] = lat[k][c];
        translations(nrm, rep);
        for (int k = 0; k < 3; k++)
            if (!periodic[k]) rep[k] = 0;
    }
    if (rep[0] < 0 || rep[1] < 0 || rep[2] < 0) return -1;
    const long long n = (long long)(2 * rep[0] + 1) * (2 * rep[1] + 1) * (2 * rep[2] + 1);
    if (n > cap) return -1;
    int t = 0;
    for (int ix = -rep[0]; ix <= rep[0]; ix++)
        for (int iy = -rep[1]; iy <= rep[1]; iy++)
            for (int iz = -rep[2]; iz <= rep[2]; iz++, t++)
                for (int c = 0; c < 3; c++) out[3 * t + c] = lat[0][c] * ix + lat[1][c] * iy + lat[2][c] * iz;
    return (int)n;
}

// Device address of the scratch array on the current device (resolved once).
cudaError_t scratch_on_current_device(unsigned char** ptr)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_ptr[dev] = static_cast<unsigned char*>(p);
    }
    *ptr = g_scratch_ptr[dev];
    return cudaSuccess;
}

}  // namespace

namespace d3 {

// Runs the pipeline; returns false and fills msg[256] on error.
bool noalloc_dispersion(const Damp& damp, int natoms, const int* numbers, const double* d_positions,
                        const double* lattice, const bool* periodic, const double* cutoffs, int precision,
                        double* d_energy, double* d_gradient, double* d_sigma, cudaStream_t stream, char* msg)
{
    auto fail = [&](const char* text) {
        std::snprintf(msg, 256, "%s", text);
        return false;
    };
    if (natoms < 1 || natoms > kNoAllocMaxAtoms) {
        std::snprintf(msg, 256, "Allocation-free evaluation supports 1 to %d atoms, got %d", kNoAllocMaxAtoms,
                      natoms);
        return false;
    }
    if (!numbers || !d_positions || !d_energy) return fail("Invalid buffers for the allocation-free evaluation");
    if (std::fabs(damp.s9) >= DBL_EPSILON)
        return fail("The allocation-free evaluation covers the two-body term only; set s9 = 0");
    if (damp.kind != kRational && damp.kind != kZero)
        return fail("The allocation-free evaluation supports the rational and zero damping");
    if (precision != DFTD3_B200_PRECISION_FP64 && precision != DFTD3_B200_PRECISION_MIXED)
        return fail("Invalid precision selector");
    for (int k = 0; k < 3 && periodic; k++)
        if (periodic[k] && !lattice) return fail("Periodic directions need a lattice");
    // a launch error still pending from earlier work would otherwise be
    // reported (and cleared) as this call's own at the end
    {
        const cudaError_t pending = cudaPeekAtLastError();
        if (pending != cudaSuccess) {
            std::snprintf(msg, 256, "CUDA error pending from earlier work: %s", cudaGetErrorString(pending));
            return false;
        }
    }

    std::lock_guard<std::mutex> lock(g_mutex);
    HostStage& h = g_host;
    // species by first occurrence and their model tables (model.f90:87-181)
    int nid = 0;
    for (int a = 0; a < natoms; a++) {
        const int z = numbers[a];
        if (z < 1 || z > D3_MAX_ELEM) return fail("Unsupported element in the allocation-free evaluation");
        int s = 0;
        while (s < nid && h.num[s] != z) s++;
        if (s == nid) {
            if (nid == kNoAllocMaxSpecies) {
                std::snprintf(msg, 256, "Allocation-free evaluation supports at most %d elements",
                              kNoAllocMaxSpecies);
                return false;
            }
            h.num[nid++] = z;
        }
        h.sp[a] = s;
        h.zeros[a] = 0;
        h.local[a] = a;
    }
    for (int s = 0; s < nid; s++) {
        const int z = h.num[s];
        h.rcov[s] = 4.0 / 3.0 * (D3_AATOAU * d3_rcov_aa[z - 1]);
        h.r4r2[s] = std::sqrt(0.5 * (d3_r4_over_r2[z - 1] * std::sqrt((double)z)));
        h.nref[s] = d3_nref[z - 1];
        for (int r = 0; r < kMaxRef; r++) h.refcn[s * kMaxRef + r] = r < h.nref[s] ? d3_refcn[(z - 1) * 7 + r] : 0.0;
    }
    for (int is = 0; is < nid; is++)
        for (int js = 0; js < nid; js++) {
            const int z1 = h.num[js], z2 = h.num[is];
            const int ic = z1 > z2 ? (z2 - 1) + z1 * (z1 - 1) / 2 : (z1 - 1) + z2 * (z2 - 1) / 2;
            h.rvdw[is * nid + js] = D3_AATOAU * d3_vdwrad_aa[ic];
        }
    std::memset(h.c6ref, 0, sizeof(double) * nid * nid * kMaxRef * kMaxRef);
    for (int is = 0; is < nid; is++)
        for (int js = 0; js < nid; js++)
            for (int ir = 0; ir < h.nref[is]; ir++)
                for (int jr = 0; jr < h.nref[js]; jr++) {
                    // get_c6(ir, jr, Z_is, Z_js), reference.f90:160-171
                    const int ati = h.num[is], atj = h.num[js];
                    double v;
                    if (ati > atj) v = d3_c6ab[((atj - 1) + ati * (ati - 1) / 2) * 49 + jr * 7 + ir];
                    else v = d3_c6ab[((ati - 1) + atj * (atj - 1) / 2) * 49 + ir * 7 + jr];
                    h.c6ref[(((size_t)is * nid + js) * kMaxRef + ir) * kMaxRef + jr] = v;
                }
    for (int k = 0; k < nid * nid * kMaxRef * kMaxRef; k++) h.c6ref_f[k] = (float)h.c6ref[k];
    for (int a = 0; a < nid; a++)
        for (int b = 0; b < nid; b++) {
            double* p = &h.pair[kPairSlots * (a * nid + b)];
            const double rrij = 3 * (h.r4r2[a] * h.r4r2[b]);   // symmetric in (a, b)
            p[0] = rrij;
            if (damp.kind == kRational) {
                const double r0 = damp.a1 * std::sqrt(rrij) + damp.a2;
                const double r02 = r0 * r0, r06 = r02 * r02 * r02;
                p[1] = r06; p[2] = r06 * r02; p[3] = r0; p[4] = std::sqrt(rrij); p[5] = 0.0;
            } else {
                const double r0 = h.rvdw[b * nid + a];
                p[1] = damp.rs6 * r0; p[2] = damp.rs8 * r0; p[3] = r0; p[4] = 0.0; p[5] = 0.0;
            }
        }
    // lattice translations per cutoff
    double lat[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    if (lattice) std::memcpy(lat, lattice, sizeof(lat));
    bool per[3];
    for (int k = 0; k < 3; k++) per[k] = periodic ? periodic[k] : (lattice != nullptr);
    Cutoffs cut;
    if (cutoffs) cut = Cutoffs{cutoffs[0], cutoffs[1], cutoffs[2], cutoffs[3], cutoffs[4]};
    const double rthr[kImageKinds] = {cut.cn, cut.disp2, cut.disp3};
    int nimg_total = 0;
    for (int k = 0; k < kImageKinds; k++) {
        const int n = lattice_points_into(lat, per, rthr[k], h.img + 3 * nimg_total, kNoAllocMaxImages);
        if (n < 0) {
            std::snprintf(msg, 256,
                          "Allocation-free evaluation supports at most %d lattice translations per cutoff "
                          "(and a non-degenerate lattice)", kNoAllocMaxImages);
            return false;
        }
        h.img_off[2 * k] = nimg_total;
        h.img_off[2 * k + 1] = nimg_total + n;
        nimg_total += n;
    }
    h.atom_off[0] = 0;
    h.atom_off[1] = natoms;

    unsigned char* base = nullptr;
    cudaError_t ce = scratch_on_current_device(&base);
    if (ce != cudaSuccess) {
        std::snprintf(msg, 256, "CUDA error resolving the scratch array: %s", cudaGetErrorString(ce));
        return false;
    }
    // carve the work arrays out of the scratch array
    const size_t n = natoms;
    Carver cv{base};
    double* x = cv.take<double>(n);
    double* y = cv.take<double>(n);
    double* z = cv.take<double>(n);
    float4* xhi = cv.take<float4>(n);
    float4* xlo = cv.take<float4>(n);
    Work w;
    w.cn = cv.take<double>(n);
    w.gw = cv.take<double>(n * kMaxRef);
    w.dgw = cv.take<double>(n * kMaxRef);
    w.gwf = cv.take<float>(n * kMaxRef);
    w.dgwf = cv.take<float>(n * kMaxRef);
    w.dEdcn = cv.take<double>(n);
    w.e_atom = cv.take<double>(n);
    w.grad = cv.take<double>(3 * n);
    w.sig_atom = cv.take<double>(kSigma * n);
    int* d_sys = cv.take<int>(n);
    int* d_local = cv.take<int>(n);
    int* d_sp = cv.take<int>(n);
    int* d_atom_off = cv.take<int>(2);
    int* d_img_off = cv.take<int>(2 * kImageKinds);
    int* d_nref = cv.take<int>(nid);
    double* d_img = cv.take<double>(3 * (size_t)nimg_total);
    double* d_rcov = cv.take<double>(nid);
    double* d_refcn = cv.take<double>((size_t)nid * kMaxRef);
    double* d_c6ref = cv.take<double>((size_t)nid * nid * kMaxRef * kMaxRef);
    float* d_c6ref_f = cv.take<float>((size_t)nid * nid * kMaxRef * kMaxRef);
    double* d_pair = cv.take<double>((size_t)nid * nid * kPairSlots);
    if (cv.overflow) return fail("Allocation-free evaluation: inputs exceed the scratch array");

    auto up = [&](void* dst, const void* src, size_t bytes) {
        return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream);
    };
    cudaError_t e = cudaSuccess;
    if (e == cudaSuccess) e = up(d_sys, h.zeros, sizeof(int) * n);
    if (e == cudaSuccess) e = up(d_local, h.local, sizeof(int) * n);
    if (e == cudaSuccess) e = up(d_sp, h.sp, sizeof(int) * n);
    if (e == cudaSuccess) e = up(d_atom_off, h.atom_off, sizeof(h.atom_off));
    if (e == cudaSuccess) e = up(d_img_off, h.img_off, sizeof(int) * 2 * kImageKinds);
    if (e == cudaSuccess) e = up(d_nref, h.nref, sizeof(int) * nid);
    if (e == cudaSuccess) e = up(d_img, h.img, sizeof(double) * 3 * nimg_total);
    if (e == cudaSuccess) e = up(d_rcov, h.rcov, sizeof(double) * nid);
    if (e == cudaSuccess) e = up(d_refcn, h.refcn, sizeof(double) * nid * kMaxRef);
    if (e == cudaSuccess) e = up(d_c6ref, h.c6ref, sizeof(double) * nid * nid * kMaxRef * kMaxRef);
    if (e == cudaSuccess) e = up(d_c6ref_f, h.c6ref_f, sizeof(float) * nid * nid * kMaxRef * kMaxRef);
    if (e == cudaSuccess) e = up(d_pair, h.pair, sizeof(double) * nid * nid * kPairSlots);
    // the host staging buffers are reused by the next call: let the copies finish
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) {
        std::snprintf(msg, 256, "CUDA error staging the allocation-free evaluation: %s", cudaGetErrorString(e));
        return false;
    }

    Batch b;
    b.nsys = 1; b.natoms = natoms; b.nid = nid;
    b.sys_of_atom = d_sys; b.atom_off = d_atom_off; b.local = d_local; b.sp = d_sp; b.ghost = nullptr;
    b.img_off = d_img_off; b.img = d_img; b.x = x; b.y = y; b.z = z; b.xhi = xhi; b.xlo = xlo;
    Species sp;
    sp.rcov = d_rcov; sp.nref = d_nref; sp.refcn = d_refcn; sp.c6ref = d_c6ref; sp.c6ref_f = d_c6ref_f;
    sp.pair = d_pair; sp.atm_r0 = nullptr;
    Config c;
    c.cut_cn = cut.cn; c.cut2 = cut.disp2; c.cut3 = cut.disp3; c.width2 = cut.width2; c.width3 = cut.width3;
    c.grad = d_gradient != nullptr || d_sigma != nullptr;
    c.mixed = precision == DFTD3_B200_PRECISION_MIXED;
    c.param_grad = false;
    Partition part;

    launch_split_positions(d_positions, natoms, x, y, z, xhi, xlo, c.mixed, stream);
    launch_coordination_number(b, sp, c, part, w, stream);
    launch_weights(b, sp, c, w, stream);
    if (std::fabs(damp.s6) >= DBL_EPSILON || std::fabs(damp.s8) >= DBL_EPSILON) {
        launch_two_body(b, sp, damp, c, part, w, stream);
    } else {
        // nothing writes these regions when the two-body term vanishes
        e = cudaMemsetAsync(w.e_atom, 0, sizeof(double) * n, stream);
        if (e == cudaSuccess && c.grad) e = cudaMemsetAsync(w.dEdcn, 0, sizeof(double) * n, stream);
        if (e == cudaSuccess && c.grad) e = cudaMemsetAsync(w.grad, 0, sizeof(double) * 3 * n, stream);
        if (e == cudaSuccess && c.grad) e = cudaMemsetAsync(w.sig_atom, 0, sizeof(double) * kSigma * n, stream);
    }
    if (e == cudaSuccess && c.grad) launch_cn_chain_rule(b, sp, c, part, w, stream);
    if (e == cudaSuccess) launch_reduce_systems(b, c, w, d_energy, d_sigma, nullptr, d_gradient, stream);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) {
        std::snprintf(msg, 256, "CUDA error in the allocation-free evaluation: %s", cudaGetErrorString(e));
        return false;
    }
    return true;
}

}  // namespace d3
