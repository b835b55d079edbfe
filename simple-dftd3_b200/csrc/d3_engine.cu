// Host-side driver of the D3 pipeline (see d3_engine.h).
#include "d3_engine.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <numeric>

#include "d3_tables.h"

namespace d3 {

namespace {

void check(cudaError_t e, const char* what)
{
    if (e != cudaSuccess)
        throw Error(std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e));
}

void cross(const double* a, const double* b, double* c)
{
    // cutoff.f90:229-238
    const double x = a[1] * b[2] - b[1] * a[2];
    const double y = a[2] * b[0] - b[2] * a[0];
    const double z = a[0] * b[1] - b[0] * a[1];
    c[0] = x; c[1] = y; c[2] = z;
}

void translations(const double lat[3][3], double rthr, int rep[3])
{
    // get_translations, cutoff.f90:204-227 (lat[k] is lattice vector k)
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
        rep[k] = (int)std::ceil(std::fabs(rthr / cs));
    }
}

double shift_back_abc(double in)
{
    // utils.f90:48-64
    const double eps = 1.0e-14;
    double out = in;
    if (in < -eps) out = in + std::ceil(-in);
    if (in > 1.0 + eps) out = in - std::floor(in);
    if (std::fabs(in - 1.0) < eps) out = in - 1.0;
    return out;
}

double covalent_radius(int z)
{
    // D3 covalent radius in Bohr, 4/3 of the tabulated radius (see d3_tables.h)
    return 4.0 / 3.0 * (D3_AATOAU * d3_rcov_aa[z - 1]);
}

double r4r2_value(int z)
{
    // data/r4r2.f90:69-70
    return std::sqrt(0.5 * (d3_r4_over_r2[z - 1] * std::sqrt((double)z)));
}

double vdw_rad(int z1, int z2)
{
    // data/vdwrad.f90:1163-1197, both elements inside the table
    const int ic = z1 > z2 ? (z2 - 1) + z1 * (z1 - 1) / 2 : (z1 - 1) + z2 * (z2 - 1) / 2;
    return D3_AATOAU * d3_vdwrad_aa[ic];
}

double ref_c6(int iref, int jref, int ati, int atj)
{
    // get_c6, reference.f90:160-171
    if (ati > atj) {
        const int ic = (atj - 1) + ati * (ati - 1) / 2;
        return d3_c6ab[ic * 49 + jref * 7 + iref];
    }
    const int ic = (ati - 1) + atj * (atj - 1) / 2;
    return d3_c6ab[ic * 49 + iref * 7 + jref];
}

}  // namespace

std::vector<double> lattice_points(const double* lattice, const bool* periodic, double rthr)
{
    const int np = (int)periodic[0] + (int)periodic[1] + (int)periodic[2];
    if (np == 0) return {0.0, 0.0, 0.0};
    double lat[3][3];
    for (int k = 0; k < 3; k++)
        for (int c = 0; c < 3; c++) lat[k][c] = lattice[3 * k + c];
    int rep[3] = {0, 0, 0};
    if (np == 3) {
        translations(lat, rthr, rep);
    } else if (np == 1) {
        for (int k = 0; k < 3; k++) {
            const double v = std::sqrt(lat[k][0] * lat[k][0] + lat[k][1] * lat[k][1] + lat[k][2] * lat[k][2]);
            rep[k] = periodic[k] ? (int)std::ceil(rthr / v) : 0;
        }
    } else {
        // get_normals, then component c of every vector is taken from the
        // lattice where periodic(c) holds (cutoff.f90:168-176)
        double nrm[3][3];
        for (int k = 0; k < 3; k++) cross(lat[(k + 1) % 3], lat[(k + 2) % 3], nrm[k]);
        for (int k = 0; k < 3; k++)
            for (int c = 0; c < 3; c++)
                if (periodic[c]) nrm[k][c] = lat[k][c];
        translations(nrm, rthr, rep);
        for (int k = 0; k < 3; k++)
            if (!periodic[k]) rep[k] = 0;
    }
    std::vector<double> t;
    t.reserve(3 * (2 * rep[0] + 1) * (2 * rep[1] + 1) * (2 * rep[2] + 1));
    for (int ix = -rep[0]; ix <= rep[0]; ix++)
        for (int iy = -rep[1]; iy <= rep[1]; iy++)
            for (int iz = -rep[2]; iz <= rep[2]; iz++)
                for (int c = 0; c < 3; c++) t.push_back(lat[0][c] * ix + lat[1][c] * iy + lat[2][c] * iz);
    return t;
}

void wrap_to_central_cell(int nat, double* xyz, const double* lattice, const bool* periodic)
{
    if (!(periodic[0] || periodic[1] || periodic[2])) return;
    // M has the lattice vectors as columns; f = M^-1 x by cofactors
    double a[3][3];
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) a[r][c] = lattice[3 * c + r];
    const double det = a[0][0] * a[1][1] * a[2][2] - a[0][0] * a[1][2] * a[2][1]
                     - a[0][1] * a[1][0] * a[2][2] + a[0][1] * a[1][2] * a[2][0]
                     + a[0][2] * a[1][0] * a[2][1] - a[0][2] * a[1][1] * a[2][0];
    const double d = 1.0 / det;
    double inv[3][3];
    inv[0][0] = +d * (a[1][1] * a[2][2] - a[1][2] * a[2][1]);
    inv[1][0] = -d * (a[1][0] * a[2][2] - a[1][2] * a[2][0]);
    inv[2][0] = +d * (a[1][0] * a[2][1] - a[1][1] * a[2][0]);
    inv[0][1] = -d * (a[0][1] * a[2][2] - a[0][2] * a[2][1]);
    inv[1][1] = +d * (a[0][0] * a[2][2] - a[0][2] * a[2][0]);
    inv[2][1] = -d * (a[0][0] * a[2][1] - a[0][1] * a[2][0]);
    inv[0][2] = +d * (a[0][1] * a[1][2] - a[0][2] * a[1][1]);
    inv[1][2] = -d * (a[0][0] * a[1][2] - a[0][2] * a[1][0]);
    inv[2][2] = +d * (a[0][0] * a[1][1] - a[0][1] * a[1][0]);
    for (int i = 0; i < nat; i++) {
        double* x = xyz + 3 * i;
        double f[3];
        for (int r = 0; r < 3; r++) f[r] = shift_back_abc(inv[r][0] * x[0] + inv[r][1] * x[1] + inv[r][2] * x[2]);
        for (int r = 0; r < 3; r++) x[r] = a[r][0] * f[0] + a[r][1] * f[1] + a[r][2] * f[2];
    }
}

bool has_overlapping_atoms(int nat, const double* xyz)
{
    // Sort by x and compare within a 1e-9 window: the same pairs as the
    // reference's O(N^2) scan report.
    std::vector<int> idx(nat);
    std::iota(idx.begin(), idx.end(), 0);
    std::sort(idx.begin(), idx.end(), [&](int a, int b) { return xyz[3 * a] < xyz[3 * b]; });
    for (int a = 0; a < nat; a++) {
        const double* p = xyz + 3 * idx[a];
        for (int b = a + 1; b < nat; b++) {
            const double* q = xyz + 3 * idx[b];
            if (q[0] - p[0] >= 1.0e-9) break;
            const double dx = q[0] - p[0], dy = q[1] - p[1], dz = q[2] - p[2];
            if (std::sqrt(dx * dx + dy * dy + dz * dz) < 1.0e-9) return true;
        }
    }
    return false;
}

template <class T>
T* Engine::dev_alloc(size_t n)
{
    void* p = nullptr;
    if (n == 0) n = 1;
    check(cudaMalloc(&p, n * sizeof(T)), "cudaMalloc");
    allocations_.push_back(p);
    alloc_epoch_++;   // captured graphs hold device pointers
    return static_cast<T*>(p);
}

Engine::Engine(int nsys, const int* natoms, const int* numbers, const double* lattices,
               const bool* periodic, int device)
{
    if (nsys <= 0) throw Error("Invalid number of systems");
    if (device < 0) check(cudaGetDevice(&device_), "cudaGetDevice");
    else device_ = device;
    check(cudaSetDevice(device_), "cudaSetDevice");
    nsys_ = nsys;
    atom_off_.assign(nsys + 1, 0);
    for (int s = 0; s < nsys; s++) {
        if (natoms[s] < 0) throw Error("Invalid number of atoms");
        atom_off_[s + 1] = atom_off_[s] + natoms[s];
        max_sys_atoms_ = std::max(max_sys_atoms_, natoms[s]);
    }
    natoms_ = atom_off_[nsys];
    sys_of_atom_.resize(natoms_);
    local_.resize(natoms_);
    for (int s = 0; s < nsys; s++)
        for (int a = atom_off_[s]; a < atom_off_[s + 1]; a++) {
            sys_of_atom_[a] = s;
            local_[a] = a - atom_off_[s];
        }
    lat_.assign(9 * (size_t)nsys, 0.0);
    per_.reset(new bool[3 * (size_t)nsys]);
    for (int s = 0; s < nsys; s++)
        for (int k = 0; k < 3; k++) per_[3 * s + k] = periodic ? periodic[3 * s + k] : (lattices != nullptr);
    if (lattices) std::copy(lattices, lattices + 9 * (size_t)nsys, lat_.begin());
    build_tables(numbers);
    ghost_.assign(natoms_, 0);

    check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate");
    check(cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, device_), "attribute");
    const int nid = tab_.nid();
    d_sys_of_atom_ = dev_alloc<int>(natoms_);
    d_atom_off_ = dev_alloc<int>(nsys + 1);
    d_local_ = dev_alloc<int>(natoms_);
    d_sp_ = dev_alloc<int>(natoms_);
    d_zid_ = dev_alloc<int>(natoms_);
    d_ghost_ = dev_alloc<uint8_t>(natoms_);
    d_img_off_ = dev_alloc<int>(kImageKinds * (nsys + 1));
    d_rcov_ = dev_alloc<double>(nid);
    d_nref_ = dev_alloc<int>(nid);
    d_refcn_ = dev_alloc<double>(nid * kMaxRef);
    d_c6ref_ = dev_alloc<double>((size_t)nid * nid * kMaxRef * kMaxRef);
    d_c6ref_f_ = dev_alloc<float>((size_t)nid * nid * kMaxRef * kMaxRef);
    d_pair_ = dev_alloc<double>((size_t)nid * nid * kPairSlots);
    d_atm_r0_ = dev_alloc<double>((size_t)nid * nid);
    d_counts_ = dev_alloc<unsigned long long>(3);
    auto up = [&](void* dst, const void* src, size_t bytes) {
        if (bytes) check(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream_), "upload");
    };
    up(d_sys_of_atom_, sys_of_atom_.data(), sizeof(int) * natoms_);
    up(d_atom_off_, atom_off_.data(), sizeof(int) * (nsys + 1));
    up(d_local_, local_.data(), sizeof(int) * natoms_);
    up(d_sp_, sp_.data(), sizeof(int) * natoms_);
    up(d_zid_, zid_.data(), sizeof(int) * natoms_);
    up(d_ghost_, ghost_.data(), natoms_);
    up(d_rcov_, tab_.rcov.data(), sizeof(double) * nid);
    up(d_nref_, tab_.nref.data(), sizeof(int) * nid);
    up(d_refcn_, tab_.refcn.data(), sizeof(double) * nid * kMaxRef);
    up(d_c6ref_, tab_.c6ref.data(), sizeof(double) * tab_.c6ref.size());
    up(d_c6ref_f_, tab_.c6ref_f.data(), sizeof(float) * tab_.c6ref_f.size());
    std::vector<double> r0((size_t)nid * nid);
    for (int a = 0; a < nid; a++)
        for (int b = 0; b < nid; b++) r0[a * nid + b] = 4.0 / 3.0 * tab_.rvdw[a * nid + b];
    up(d_atm_r0_, r0.data(), sizeof(double) * r0.size());
    // tiles of 32 consecutive atoms of a system
    std::vector<int> tile_off(nsys + 1, 0), tile_sys;
    for (int sy = 0; sy < nsys; sy++) {
        const int nt = (natoms[sy] + kTile - 1) / kTile;
        tile_off[sy + 1] = tile_off[sy] + nt;
        for (int t = 0; t < nt; t++) tile_sys.push_back(sy);
    }
    ntiles_ = tile_off[nsys];
    // two-body units: tile pairs (it >= jt) of each system
    std::vector<int2> units;
    std::vector<int> unit_base(nsys, 0);
    for (int sy = 0; sy < nsys; sy++) {
        unit_base[sy] = (int)units.size();
        const int nt = tile_off[sy + 1] - tile_off[sy];
        for (int it = 0; it < nt; it++)
            for (int jt = 0; jt <= it; jt++) units.push_back(make_int2(tile_off[sy] + it, tile_off[sy] + jt));
    }
    pu_.nunits = (int)units.size();
    d_units_ = dev_alloc<int2>(std::max<size_t>(units.size(), 1));
    d_unit_base_ = dev_alloc<int>(nsys);
    up(d_units_, units.data(), sizeof(int2) * units.size());
    up(d_unit_base_, unit_base.data(), sizeof(int) * nsys);
    pu_.units = d_units_;
    pu_.unit_base = d_unit_base_;
    pu_.U = dev_alloc<double>(species_vector_doubles(natoms_, nid));
    pu_.unit_i = dev_alloc<double>((size_t)std::max(pu_.nunits, 1) * pair_unit_slot_doubles());
    pu_.unit_j = pu_.unit_i + (size_t)std::max(pu_.nunits, 1) * pair_unit_i_doubles();
    d_tile_off_ = dev_alloc<int>(nsys + 1);
    d_tile_sys_ = dev_alloc<int>(std::max(ntiles_, 1));
    up(d_tile_off_, tile_off.data(), sizeof(int) * (nsys + 1));
    up(d_tile_sys_, tile_sys.data(), sizeof(int) * ntiles_);
    // three-body dense blocks per system
    c6mat_off_.assign(nsys, 0);
    long long off = 0;
    for (int s = 0; s < nsys; s++) {
        c6mat_off_[s] = off;
        off += (long long)natoms[s] * natoms[s];
    }
    c6mat_total_ = off;
    sys_natoms_.assign(natoms, natoms + nsys);
    auto_split_ = 1;
    for (int sy = 0; sy < nsys; sy++)
        if (per_[3 * sy] || per_[3 * sy + 1] || per_[3 * sy + 2]) auto_split_ = 2;
    any_periodic_ = auto_split_ == 2;
    d_mol_order_ = dev_alloc<int>(nsys);
    d_sys_mol_ = dev_alloc<uint8_t>(nsys);
    configure_molecules();
    check(cudaStreamSynchronize(stream_), "upload sync");
}

Engine::~Engine()
{
    cudaSetDevice(device_);
    if (stream_) cudaStreamSynchronize(stream_);
    for (auto& e : ev_)
        if (e) cudaEventDestroy(e);
    for (auto& e : kev_)
        if (e) cudaEventDestroy(e);
    if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
    for (void* p : allocations_) cudaFree(p);
    if (h_stage_) cudaFreeHost(h_stage_);
    if (h_atm_counts_) cudaFreeHost(h_atm_counts_);
    if (h_guard_) cudaFreeHost(h_guard_);
    if (stream_) cudaStreamDestroy(stream_);
}

void Engine::configure_molecules()
{
    // molecules for the block-per-system three-body kernel: no periodic
    // direction and at most atm_mol_max_atoms() atoms, largest first
    std::vector<uint8_t> is_mol(nsys_, 0);
    mol_order_.clear();
    root_atoms_ = 0;
    for (int s = 0; s < nsys_; s++) {
        const bool per_any = per_[3 * s] || per_[3 * s + 1] || per_[3 * s + 2];
        if (tune_.atm_mol != 2 && !per_any && sys_natoms_[s] <= atm_mol_max_atoms()) mol_order_.push_back(s);
        else root_atoms_ += sys_natoms_[s];
    }
    // one block per molecule pays off for many molecules; a few are spread
    // over all SMs by the neighbour-list kernel instead
    if (tune_.atm_mol == 0 && (int)mol_order_.size() < sms_) {
        for (int sy : mol_order_) root_atoms_ += sys_natoms_[sy];
        mol_order_.clear();
    }
    std::stable_sort(mol_order_.begin(), mol_order_.end(),
                     [&](int a, int b) { return sys_natoms_[a] > sys_natoms_[b]; });
    for (int sy : mol_order_) is_mol[sy] = 1;
    check(cudaStreamSynchronize(stream_), "molecules");
    if (!mol_order_.empty())
        check(cudaMemcpy(d_mol_order_, mol_order_.data(), sizeof(int) * mol_order_.size(), cudaMemcpyHostToDevice),
              "molecule order");
    check(cudaMemcpy(d_sys_mol_, is_mol.data(), nsys_, cudaMemcpyHostToDevice), "molecule flags");
}

void Engine::build_tables(const int* numbers)
{
    // species by first occurrence over the batch
    sp_.resize(natoms_);
    for (int a = 0; a < natoms_; a++) {
        const int z = numbers[a];
        if (z < 1 || z > D3_MAX_ELEM) throw Error("Unsupported element with atomic number " + std::to_string(z));
        auto it = std::find(tab_.num.begin(), tab_.num.end(), z);
        if (it == tab_.num.end()) {
            tab_.num.push_back(z);
            sp_[a] = tab_.nid() - 1;
        } else {
            sp_[a] = (int)(it - tab_.num.begin());
        }
    }
    // species by first occurrence inside each system, from 1: the species
    // index mol%id of a structure of its own (used by the Z damping)
    zid_.resize(natoms_);
    for (size_t sy = 0; sy + 1 < atom_off_.size(); sy++) {
        std::vector<int> seen;
        for (int a = atom_off_[sy]; a < atom_off_[sy + 1]; a++) {
            auto it = std::find(seen.begin(), seen.end(), numbers[a]);
            if (it == seen.end()) {
                seen.push_back(numbers[a]);
                zid_[a] = (int)seen.size();
            } else {
                zid_[a] = (int)(it - seen.begin()) + 1;
            }
        }
    }
    const int nid = tab_.nid();
    tab_.rcov.resize(nid);
    tab_.r4r2.resize(nid);
    tab_.nref.resize(nid);
    tab_.refcn.assign((size_t)nid * kMaxRef, 0.0);
    for (int s = 0; s < nid; s++) {
        const int z = tab_.num[s];
        tab_.rcov[s] = covalent_radius(z);
        tab_.r4r2[s] = r4r2_value(z);
        tab_.nref[s] = d3_nref[z - 1];
        for (int r = 0; r < tab_.nref[s]; r++) tab_.refcn[s * kMaxRef + r] = d3_refcn[(z - 1) * 7 + r];
    }
    tab_.rvdw.assign((size_t)nid * nid, 0.0);
    for (int is = 0; is < nid; is++)
        for (int js = 0; js <= is; js++) {
            const double r = vdw_rad(tab_.num[js], tab_.num[is]);
            tab_.rvdw[js * nid + is] = r;
            tab_.rvdw[is * nid + js] = r;
        }
    // c6(ir, jr, is, js) as filled by new_d3_model (model.f90:150-163)
    tab_.c6ref.assign((size_t)nid * nid * kMaxRef * kMaxRef, 0.0);
    auto at = [&](int ir, int jr, int is, int js) -> double& {
        return tab_.c6ref[(((size_t)is * nid + js) * kMaxRef + ir) * kMaxRef + jr];
    };
    for (int is = 0; is < nid; is++)
        for (int js = 0; js <= is; js++)
            for (int ir = 0; ir < tab_.nref[is]; ir++)
                for (int jr = 0; jr < tab_.nref[js]; jr++) {
                    at(jr, ir, js, is) = ref_c6(jr, ir, tab_.num[js], tab_.num[is]);
                    at(ir, jr, is, js) = at(jr, ir, js, is);
                }
    tab_.c6ref_f.assign(tab_.c6ref.begin(), tab_.c6ref.end());
}

bool Engine::periodic_any(int sys) const
{
    return per_[3 * sys] || per_[3 * sys + 1] || per_[3 * sys + 2];
}

void Engine::set_ghost(const std::vector<uint8_t>& ghost)
{
    ghost_ = ghost;
    ghost_.resize(natoms_, 0);
    check(cudaMemcpyAsync(d_ghost_, ghost_.data(), natoms_, cudaMemcpyHostToDevice, stream_), "ghost");
    check(cudaStreamSynchronize(stream_), "ghost sync");
}

void Engine::set_partition(int part, int nparts, bool cn_partitioned)
{
    part_.part = part;
    part_.nparts = nparts;
    cn_partitioned_ = cn_partitioned;
}

void Engine::set_lattices(const double* lattices)
{
    if (!lattices) return;
    if (!std::equal(lattices, lattices + 9 * (size_t)nsys_, lat_.begin())) {
        std::copy(lattices, lattices + 9 * (size_t)nsys_, lat_.begin());
        images_valid_ = false;
    }
}

void Engine::counts(long long out[3]) const
{
    unsigned long long h[3] = {0, 0, 0};
    check(cudaMemcpy(h, d_counts_, sizeof(h), cudaMemcpyDeviceToHost), "counts");
    for (int k = 0; k < 3; k++) out[k] = (long long)h[k];
}

void Engine::ensure_images(cudaStream_t stream)
{
    if (images_valid_) return;
    const double rthr[kImageKinds] = {cut_.cn, cut_.disp2, cut_.disp3};
    std::vector<int> off(kImageKinds * (nsys_ + 1), 0);
    std::vector<double> all;
    for (int k = 0; k < kImageKinds; k++) {
        for (int s = 0; s < nsys_; s++) {
            off[k * (nsys_ + 1) + s] = (int)(all.size() / 3);
            std::vector<double> t = lattice_points(&lat_[9 * s], &per_[3 * s], rthr[k]);
            all.insert(all.end(), t.begin(), t.end());
        }
        off[k * (nsys_ + 1) + nsys_] = (int)(all.size() / 3);
    }
    if (all.size() > img_capacity_) {
        if (d_img_) {
            check(cudaStreamSynchronize(stream), "images sync");
            auto it = std::find(allocations_.begin(), allocations_.end(), (void*)d_img_);
            if (it != allocations_.end()) allocations_.erase(it);
            check(cudaFree(d_img_), "cudaFree");
            alloc_epoch_++;
        }
        img_capacity_ = all.size() + all.size() / 4 + 3;
        d_img_ = dev_alloc<double>(img_capacity_);
    }
    check(cudaMemcpyAsync(d_img_, all.data(), sizeof(double) * all.size(), cudaMemcpyHostToDevice, stream), "images");
    check(cudaMemcpyAsync(d_img_off_, off.data(), sizeof(int) * off.size(), cudaMemcpyHostToDevice, stream), "img_off");
    img_off_host_ = off;
    // the host vectors go out of scope: make the copies complete first
    check(cudaStreamSynchronize(stream), "images sync");
    images_valid_ = true;
}

void Engine::ensure_workspace(bool grad, bool param_grad, bool threebody)
{
    if (!ws_ready_) {
        const size_t n = natoms_;
        d_x_ = dev_alloc<double>(n); d_y_ = dev_alloc<double>(n); d_z_ = dev_alloc<double>(n);
        d_keys_in_ = dev_alloc<unsigned long long>(n);
        d_keys_out_ = dev_alloc<unsigned long long>(n);
        d_idx_in_ = dev_alloc<int>(n);
        d_perm_ = dev_alloc<int>(n);
        d_identity_ = dev_alloc<int>(n);
        {
            std::vector<int> id(n);
            std::iota(id.begin(), id.end(), 0);
            check(cudaMemcpy(d_identity_, id.data(), sizeof(int) * n, cudaMemcpyHostToDevice), "identity order");
        }
        d_sp_sorted_ = dev_alloc<int>(n);
        d_local_sorted_ = dev_alloc<int>(n);
        d_zid_sorted_ = dev_alloc<int>(n);
        d_ghost_sorted_ = dev_alloc<uint8_t>(n);
        d_tiles_ = dev_alloc<double4>(std::max(ntiles_, 1));
        d_shape_ = dev_alloc<int2>(std::max(nsys_, 1));
        sort_bytes_ = sort_temp_bytes(natoms_);
        d_sort_temp_ = dev_alloc<unsigned char>(sort_bytes_);
        d_xhi_ = dev_alloc<float4>(n); d_xlo_ = dev_alloc<float4>(n);
        work_.cn = dev_alloc<double>(n);
        work_.gw = dev_alloc<double>(n * kMaxRef);
        work_.dgw = dev_alloc<double>(n * kMaxRef);
        work_.gwf = dev_alloc<float>(n * kMaxRef);
        work_.dgwf = dev_alloc<float>(n * kMaxRef);
        work_.dEdcn = dev_alloc<double>(n);
        work_.e_atom = dev_alloc<double>(n);
        work_.grad = dev_alloc<double>(3 * n);
        work_.sig_atom = dev_alloc<double>(kSigma * n);
        work_.cn_sig = dev_alloc<double>(kSigma * n);
        d_pos_in_ = dev_alloc<double>(3 * n);
        // energies, gradient and virials side by side: one copy to the host
        d_energies_ = dev_alloc<double>(nsys_ + 3 * n + 9 * (size_t)nsys_);
        d_grad_out_ = d_energies_ + nsys_;
        d_sigma_ = d_grad_out_ + 3 * n;
        ws_ready_ = true;
    }
    if (param_grad && !ws_pg_) {
        work_.pg_atom = dev_alloc<double>(kParamGrad * (size_t)natoms_);
        d_pg_out_ = dev_alloc<double>(kParamGrad * (size_t)nsys_);
        ws_pg_ = true;
    }
    if (!h_guard_) {
        check(cudaMallocHost(&h_guard_, sizeof(int)), "cudaMallocHost");
        *h_guard_ = 0;
    }
    (void)grad;
    (void)threebody;
}

void Engine::upload_pair_table(const Damp& d, cudaStream_t stream)
{
    if (pair_valid_ && std::memcmp(&d, &last_damp_, sizeof(Damp)) == 0) return;
    const int nid = tab_.nid();
    std::vector<double> t((size_t)nid * nid * kPairSlots, 0.0);
    for (int a = 0; a < nid; a++)
        for (int b = 0; b < nid; b++) {
            double* p = &t[kPairSlots * (a * nid + b)];
            // rrij = 3 r4r2_i r4r2_j (rational.f90:458, zero.f90:475), the product
            // formed first so that the (a, b) and (b, a) entries are equal and a
            // pair's value does not depend on which atom comes first
            const double rrij = 3 * (tab_.r4r2[a] * tab_.r4r2[b]);
            p[0] = rrij;
            switch (d.kind) {
            case kRational: {
                const double r0 = d.a1 * std::sqrt(rrij) + d.a2;
                const double r02 = r0 * r0;
                const double r06 = r02 * r02 * r02;
                p[1] = r06;
                p[2] = r06 * r02;
                p[3] = r0;
                p[4] = std::sqrt(rrij);
                break;
            }
            case kZero: {
                const double r0 = tab_.rvdw[b * nid + a];
                p[1] = d.rs6 * r0;
                p[2] = d.rs8 * r0;
                p[3] = r0;
                break;
            }
            case kMZero: {   // mzero.f90:441-447
                const double r0 = tab_.rvdw[b * nid + a];
                p[1] = 1.0 / (d.rs6 * r0);
                p[2] = 1.0 / (d.rs8 * r0);
                p[3] = d.bet * r0;
                p[4] = d.rs6 * d.bet * r0 * r0;
                p[5] = d.rs8 * d.bet * r0 * r0;
                break;
            }
            case kOptimizedPower: {   // optimizedpower.f90:421-429
                const double r0 = d.a1 * std::sqrt(rrij) + d.a2;
                const double r02 = r0 * r0;
                const double r06 = r02 * r02 * r02;
                const double ab = std::pow(r0, d.bet);
                p[1] = ab * r06;
                p[2] = ab * r06 * r02;
                break;
            }
            case kCSO: {   // cso.f90:421-426 with a3 = rs6, a4 = rs8
                const double r0 = std::sqrt(rrij);
                p[1] = std::pow(d.rs6 * r0 + d.rs8, 6);
                p[2] = d.a2 * r0;
                break;
            }
            default:       // Z damping: the constant depends on the atoms' species indices
                break;
            }
        }
    check(cudaMemcpyAsync(d_pair_, t.data(), sizeof(double) * t.size(), cudaMemcpyHostToDevice, stream), "pair table");
    check(cudaStreamSynchronize(stream), "pair table sync");
    last_damp_ = d;
    pair_valid_ = true;
}

bool Engine::cn_single_chunk() const
{
    // every system's CN lattice points within one chunk of the tile sweep
    if (img_off_host_.empty()) return false;
    for (int sy = 0; sy < nsys_; sy++) {
        const int k0 = img_off_host_[kImgCN * (nsys_ + 1) + sy], k1 = img_off_host_[kImgCN * (nsys_ + 1) + sy + 1];
        if (k1 - k0 > kCnStoreChunk) return false;
    }
    return true;
}

void Engine::make_views(Batch& b, Species& s) const
{
    b.nsys = nsys_; b.natoms = natoms_; b.nid = tab_.nid();
    b.sys_of_atom = d_sys_of_atom_; b.atom_off = d_atom_off_; b.local = d_local_sorted_; b.sp = d_sp_sorted_;
    b.zid = d_zid_sorted_;
    b.ghost = d_ghost_sorted_; b.img_off = d_img_off_; b.img = d_img_;
    b.x = d_x_; b.y = d_y_; b.z = d_z_; b.xhi = d_xhi_; b.xlo = d_xlo_;
    b.perm = d_perm_; b.tiles = d_tiles_; b.tile_off = d_tile_off_; b.tile_sys = d_tile_sys_;
    s.rcov = d_rcov_; s.nref = d_nref_; s.refcn = d_refcn_; s.c6ref = d_c6ref_;
    s.c6ref_f = d_c6ref_f_; s.pair = d_pair_; s.atm_r0 = d_atm_r0_;
}

// Spatial order of the atoms, the sorted atom arrays and the tile bounds.
void Engine::order_atoms(const Damp& d, const double* d_positions, const Batch& b, bool mixed, cudaStream_t stream)
{
    const int* zid_in = d.kind == kZDamping ? d_zid_ : nullptr;
    // one block per system pays off for many systems; a few large ones are
    // ordered faster by the rank passes, which spread each system over all SMs
    if (!(tune_.morton_cell > 0.0) && max_sys_atoms_ <= kOrderBlockMax && nsys_ >= kOrderBlockMinSystems) {
        launch_order_block(d_positions, nsys_, max_sys_atoms_, d_atom_off_, d_tile_off_, d_sp_, d_ghost_, zid_in,
                           mixed, d_perm_, d_x_, d_y_, d_z_, d_xhi_, d_xlo_, d_sp_sorted_, d_ghost_sorted_,
                           d_local_sorted_, d_zid_sorted_, d_tiles_, stream);
        return;
    }
    if (!(tune_.morton_cell > 0.0) && max_sys_atoms_ <= kRankOrderMax) {
        launch_rank_order(d_positions, natoms_, nsys_, max_sys_atoms_, d_sys_of_atom_, d_atom_off_, d_tile_off_,
                          d_shape_, d_keys_in_, d_keys_out_, d_sp_, d_ghost_, zid_in, mixed, d_perm_, d_x_, d_y_,
                          d_z_, d_xhi_, d_xlo_, d_sp_sorted_, d_ghost_sorted_, d_local_sorted_, d_zid_sorted_,
                          stream);
    } else {
        launch_spatial_sort(d_positions, natoms_, d_sys_of_atom_, tune_.morton_cell > 0.0 ? tune_.morton_cell : 3.0,
                            d_keys_in_, d_keys_out_, d_idx_in_, d_perm_, d_sort_temp_, sort_bytes_, stream);
        launch_gather_sorted(d_positions, d_perm_, d_sp_, d_ghost_, d_sys_of_atom_, d_atom_off_, natoms_, d_x_, d_y_,
                             d_z_, d_xhi_, d_xlo_, d_sp_sorted_, d_ghost_sorted_, d_local_sorted_, mixed, stream,
                             zid_in, d_zid_sorted_);
    }
    launch_tile_bounds(b, d_tile_sys_, ntiles_, d_tiles_, stream);
}

void Engine::pairwise_host(const Damp& d, const double* positions, double* energy2, double* energy3)
{
    check(cudaSetDevice(device_), "cudaSetDevice");
    cudaStream_t stream = stream_;
    ensure_images(stream);
    ensure_workspace(false, false, false);
    upload_pair_table(d, stream);
    const long long total = std::max<long long>(c6mat_total_, 1);
    if (!d_pw_) {
        d_pw_ = dev_alloc<double>(3 * (size_t)total);
        d_pw_off_ = dev_alloc<long long>(nsys_);
        check(cudaMemcpy(d_pw_off_, c6mat_off_.data(), sizeof(long long) * nsys_, cudaMemcpyHostToDevice),
              "pairwise offsets");
    }
    check(cudaMemcpyAsync(d_pos_in_, positions, sizeof(double) * 3 * natoms_, cudaMemcpyHostToDevice, stream),
          "positions");
    Batch b;
    Species s;
    make_views(b, s);
    Config c;
    c.cut_cn = cut_.cn; c.cut2 = cut_.disp2; c.cut3 = cut_.disp3;
    c.width2 = cut_.width2; c.width3 = cut_.width3;
    c.grad = false; c.mixed = false; c.param_grad = false; c.cn_partitioned = false;
    Work w = work_;
    w.counts = nullptr; w.e3_atom = nullptr; w.sig3_atom = nullptr; w.pg_atom = nullptr;
    pu_.split = cn_split();
    pu_.cn_store = nullptr;
    pu_.cn_store_ok = nullptr;
    order_atoms(d, d_pos_in_, b, false, stream);
    launch_cn_units(b, s, c, Partition{}, w, pu_, false, stream);
    launch_weights(b, s, c, w, stream);
    launch_pairwise(b, s, d, c, w, d_pw_off_, c6mat_total_, d_pw_, d_pw_ + total, d_pw_ + 2 * total, stream);
    check(cudaGetLastError(), "pairwise kernels");
    check(cudaMemcpyAsync(energy2, d_pw_ + total, sizeof(double) * c6mat_total_, cudaMemcpyDeviceToHost, stream),
          "pairwise energy2");
    check(cudaMemcpyAsync(energy3, d_pw_ + 2 * total, sizeof(double) * c6mat_total_, cudaMemcpyDeviceToHost, stream),
          "pairwise energy3");
    check(cudaStreamSynchronize(stream), "pairwise");
}

// Items per tile pair with tuning 0 (measured on B200): one for batches of
// molecules; for periodic systems two, and for the CN sweeps of the mixed
// form one once the units alone give every SM eight warps.
int Engine::pair_split() const
{
    if (tune_.pair_split) return tune_.pair_split;
    return auto_split_ == 1 ? 1 : 2;
}

int Engine::cn_split() const
{
    if (tune_.pair_split) return tune_.pair_split;
    if (auto_split_ == 1) return 1;
    return mixed_ && pu_.nunits >= 8 * sms_ ? 1 : 2;
}

void Engine::hessian_host(const Damp& d, const double* positions, double* hessian)
{
    if (nsys_ != 1) throw Error("The Hessian is evaluated for one structure at a time");
    check(cudaSetDevice(device_), "cudaSetDevice");
    cudaStream_t stream = stream_;
    ensure_images(stream);
    ensure_workspace(false, false, false);
    upload_pair_table(d, stream);
    const int n = natoms_;
    const size_t nh = 9 * (size_t)n * n;
    if (!d_hs_) {
        d_hs_ = dev_alloc<double>(hessian_scratch_doubles(n) + nh);
        const int nid = tab_.nid();
        d_rvdw_ = dev_alloc<double>((size_t)nid * nid);
        check(cudaMemcpy(d_rvdw_, tab_.rvdw.data(), sizeof(double) * nid * nid, cudaMemcpyHostToDevice), "rvdw");
    }
    check(cudaMemcpyAsync(d_pos_in_, positions, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, stream), "positions");
    Batch b;
    Species s;
    make_views(b, s);
    Config c;
    c.cut_cn = cut_.cn; c.cut2 = cut_.disp2; c.cut3 = cut_.disp3;
    c.width2 = cut_.width2; c.width3 = cut_.width3;
    c.grad = true; c.mixed = false;
    const int range[6] = {img_off_host_[kImgCN * 2], img_off_host_[kImgCN * 2 + 1], img_off_host_[kImgDisp2 * 2],
                          img_off_host_[kImgDisp2 * 2 + 1], img_off_host_[kImgDisp3 * 2],
                          img_off_host_[kImgDisp3 * 2 + 1]};
    double* H = d_hs_ + hessian_scratch_doubles(n);
    launch_hessian(s, d, c, part_, n, tab_.nid(), d_pos_in_, d_sp_, d_zid_, d_ghost_, d_img_, range, d_rvdw_, d_hs_,
                   H, stream);
    check(cudaGetLastError(), "hessian kernels");
    check(cudaMemcpyAsync(hessian, H, sizeof(double) * nh, cudaMemcpyDeviceToHost, stream), "hessian");
    check(cudaStreamSynchronize(stream), "hessian");
}

// The direct path (d3_kernels.cu: one warp per atom over its partners, atoms
// in input order) for batches of small systems, where the tile sweeps are
// latency-bound: rational or zero damping, no work partition, reducer,
// parameter derivatives or term counters.
bool Engine::direct_pairs(const Damp& d, bool pg) const
{
    if (reducer_ || counting_ || pg || part_.nparts > 1) return false;
    if (d.kind != kRational && d.kind != kZero) return false;
    return max_sys_atoms_ <= kDirectMaxAtoms && natoms_ <= kDirectMaxTotal;
}

void Engine::run(const Damp& d, const double* d_positions, double* d_energies, double* d_gradient,
                 double* d_sigma9, double* d_param_grad, bool grad, cudaStream_t stream)
{
    const bool pg = d_param_grad != nullptr;
    if (pg && !damping_has_param_grad(d.kind))
        throw Error("Damping parameter derivatives are available for the rational and zero damping only");
    const bool threebody = std::fabs(d.s9) >= DBL_EPSILON;
    ensure_images(stream);
    ensure_workspace(grad, pg, threebody);
    upload_pair_table(d, stream);

    Batch b;
    Species s;
    make_views(b, s);
    Config c;
    c.cut_cn = cut_.cn; c.cut2 = cut_.disp2; c.cut3 = cut_.disp3;
    c.width2 = cut_.width2; c.width3 = cut_.width3;
    c.grad = grad; c.mixed = mixed_; c.param_grad = pg; c.cn_partitioned = cn_partitioned_;
    // the CN sweeps and the two-body sweep split the tile pairs each their own way
    pu_.split = pair_split();
    // molecules: the two-body diagonal walk (FP64 only for systems of at most
    // 256 atoms, where few tile pairs lie beyond the cutoff)
    pu_.single_image = !any_periodic_ && (mixed_ || max_sys_atoms_ <= 256);
    PairUnits pcn = pu_;
    pcn.split = cn_split();
    // the CN pass keeps the chain rule's per-pair sums when every system's CN
    // translations fit one chunk and the buffer stays below kCnStoreCap
    pcn.cn_store = nullptr;
    pcn.cn_store_ok = nullptr;
    if (grad && cn_single_chunk()) {
        const size_t bytes = cn_store_bytes(pcn, mixed_);
        if (bytes <= kCnStoreCap && (bytes <= cn_store_cap_ || !capturing_)) {
            if (bytes > cn_store_cap_) {
                free_block(d_cn_store_);
                void* ok = d_cn_store_ok_;
                free_block(ok);
                d_cn_store_ = dev_alloc<unsigned char>(bytes);
                d_cn_store_ok_ = dev_alloc<unsigned char>((size_t)pu_.nunits * 4);
                cn_store_cap_ = bytes;
            }
            pcn.cn_store = d_cn_store_;
            pcn.cn_store_ok = d_cn_store_ok_;
        }
    }
    Work w = work_;
    w.counts = counting_ ? d_counts_ : nullptr;
    w.e3_atom = nullptr;
    w.sig3_atom = nullptr;
    if (!pg) w.pg_atom = nullptr;
    if (counting_) check(cudaMemsetAsync(d_counts_, 0, 3 * sizeof(unsigned long long), stream), "counts");

    const bool timed = profiling_ && !capturing_;
    auto mark = [&](int k) {
        if (timed) check(cudaEventRecord(ev_[k], stream), "cudaEventRecord");
    };
    if (timed && !ev_[0]) {
        for (auto& e : ev_) check(cudaEventCreate(&e), "cudaEventCreate");
        for (auto& e : kev_) check(cudaEventCreate(&e), "cudaEventCreate");
    }
    kev3_recorded_ = false;
    mark(0);
    // small systems: atoms in input order and the pair sums of each atom in one
    // warp (no ordering, tiles or slot gathers; fewer and shorter launches)
    const bool direct = direct_pairs(d, pg);
    if (direct) {
        // the input arrays are the atom arrays; the CN kernel writes the positions
        b.sp = d_sp_;
        b.ghost = d_ghost_;
        b.local = d_local_;
        b.perm = d_identity_;
        b.tiles = nullptr;
    } else {
        order_atoms(d, d_positions, b, mixed_, stream);
    }
    mark(1);
    // without a reducer the CN pass also writes the reference weights and the
    // species vectors (one kernel after the sweep instead of three); above
    // kFusedWeightsMaxAtoms atoms the separate weight and species-vector
    // kernels, with a thread per atom and per vector entry, are faster
    // (the direct path: the CN kernel itself, one warp per atom)
    const bool two_body = two_body_active(d) || pg;
    const bool fused = !reducer_ && (direct || natoms_ <= kFusedWeightsMaxAtoms);
    if (direct) {
        const InputPositions in{d_positions, d_x_, d_y_, d_z_, d_xhi_, d_xlo_};
        launch_coordination_number(b, s, c, part_, w, stream, &in, pu_.U);
    }
    else launch_cn_units(b, s, c, part_, w, pcn, false, stream, fused, fused && two_body ? pu_.U : nullptr);
    if (reducer_) reduce(w.cn, natoms_, stream);
    mark(2);
    if (!fused) launch_weights(b, s, c, w, stream);
    mark(3);
    if (two_body && direct) {
        launch_two_body(b, s, d, c, part_, w, stream, pu_.U);
    } else if (two_body) {
        launch_two_body_units(b, s, d, c, part_, w, pu_, stream, timed ? kev_[0] : nullptr, timed ? kev_[1] : nullptr,
                              fused);
    } else {
        check(cudaMemsetAsync(w.e_atom, 0, sizeof(double) * natoms_, stream), "memset");
        if (grad) {
            check(cudaMemsetAsync(w.dEdcn, 0, sizeof(double) * natoms_, stream), "memset");
            check(cudaMemsetAsync(w.grad, 0, sizeof(double) * 3 * natoms_, stream), "memset");
            check(cudaMemsetAsync(w.sig_atom, 0, sizeof(double) * kSigma * natoms_, stream), "memset");
        }
    }
    mark(4);
    species_ready_ = direct || two_body;
    if (threebody) {
        run_three_body(b, s, d, c, w, stream);
        if (pg) {
            w.e3_pg = w.e3_atom;
            w.pg_s9_scale = 1.0 / d.s9;
        }
    } else if (pg) {
        // dE/ds9 at s9 = 0: the three-body energy at unit s9, not added to the energy
        Damp d1 = d;
        d1.s9 = 1.0;
        Config c1 = c;
        c1.grad = false;
        Work w1 = w;
        run_three_body(b, s, d1, c1, w1, stream);
        w.e3_pg = w1.e3_atom;
        w.pg_s9_scale = 1.0;
    }
    mark(5);
    if (grad) {
        if (reducer_) reduce(w.dEdcn, natoms_, stream);
        if (direct) launch_cn_chain_rule(b, s, c, part_, w, stream, true);
        else launch_cn_units(b, s, c, part_, w, pcn, true, stream);
    }
    mark(6);
    if (!reducer_) {
        launch_reduce_systems(b, c, w, d_energies, d_sigma9, d_param_grad, d_gradient, stream);
    } else {
        // this part's results in one buffer, summed over the parts in one call
        double* re = d_red_;
        double* rp = re + nsys_;
        double* rs = rp + (size_t)kParamGrad * nsys_;
        double* rg = rs + 9 * (size_t)nsys_;
        launch_reduce_systems(b, c, w, re, grad ? rs : nullptr, pg ? rp : nullptr, grad ? rg : nullptr, stream);
        if (!pg) check(cudaMemsetAsync(rp, 0, sizeof(double) * kParamGrad * nsys_, stream), "memset");
        const size_t len = (size_t)nsys_ * (1 + kParamGrad) + (grad ? 9 * (size_t)nsys_ + 3 * (size_t)natoms_ : 0);
        reduce(d_red_, (int)len, stream);
        auto out = [&](double* dst, const double* src, size_t n) {
            if (dst) check(cudaMemcpyAsync(dst, src, sizeof(double) * n, cudaMemcpyDeviceToDevice, stream), "results");
        };
        out(d_energies, re, nsys_);
        out(d_param_grad, rp, (size_t)kParamGrad * nsys_);
        out(d_sigma9, rs, 9 * (size_t)nsys_);
        out(d_gradient, rg, 3 * (size_t)natoms_);
    }
    mark(7);
    if (!capturing_) ev_recorded_ = profiling_;
    check(cudaGetLastError(), "kernel launch");
}

void Engine::free_block(void*& p)
{
    if (!p) return;
    auto it = std::find(allocations_.begin(), allocations_.end(), p);
    if (it != allocations_.end()) allocations_.erase(it);
    check(cudaFree(p), "cudaFree");
    alloc_epoch_++;
    p = nullptr;
}

void Engine::run_three_body(const Batch& b, const Species& s, const Damp& d, const Config& c, Work& w,
                            cudaStream_t stream)
{
    const int n = natoms_;
    if (!atm_ready_) {
        d_c6mat_off_ = dev_alloc<long long>(nsys_);
        check(cudaMemcpy(d_c6mat_off_, c6mat_off_.data(), sizeof(long long) * nsys_, cudaMemcpyHostToDevice),
              "c6 offsets");
        // sized for the FP64 entries, which also hold the FP32 ones
        d_c6mat_ = dev_alloc<unsigned char>(atm_c6_entry_bytes(false) * (size_t)std::max<long long>(c6mat_total_, 1));
        d_cnt_ = dev_alloc<int>(n + 1);
        d_off_ = dev_alloc<long long>(n + 1);
        d_maxcnt_ = dev_alloc<int>(1);
        d_queue_ = dev_alloc<unsigned int>(2);   // root queue, molecule queue
        d_e3_ = dev_alloc<double>(n);
        d_sig3_ = dev_alloc<double>((size_t)kSigma * n);
        d_fxacc_ = dev_alloc<unsigned long long>((size_t)8 * n);
        scan_bytes_ = scan_temp_bytes(n);
        d_scan_temp_ = dev_alloc<unsigned char>(scan_bytes_);
        check(cudaMallocHost(&h_atm_counts_, 2 * sizeof(long long)), "cudaMallocHost");
        d_guard_ = dev_alloc<int>(1);
        check(cudaMemsetAsync(d_guard_, 0, sizeof(int), stream), "memset");
        atm_ready_ = true;
    }
    // the two-body pass computed the species vectors; without it they are computed here
    if (!species_ready_) launch_species_vectors(b, s, c, w, pu_.U, stream);
    launch_c6_matrix(b, s, w, pu_.U, (d.alp + 2.0) / 3.0, d_c6mat_off_, d_c6mat_, c6mat_total_, c.mixed, stream);
    if (root_atoms_ > 0) {
        check(cudaMemsetAsync(d_maxcnt_, 0, sizeof(int), stream), "memset");
        check(cudaMemsetAsync(d_cnt_ + n, 0, sizeof(int), stream), "memset");
        launch_nbr_count(b, c, d_sys_mol_, d_cnt_, d_maxcnt_, stream);
        launch_scan(d_scan_temp_, scan_bytes_, d_cnt_, d_off_, n, stream);
        const int blocks = std::max(1, std::min(n, sms_ * atm_blocks(c.mixed, c.grad)));
        int stride = atm_stride_;
        if (!capturing_) {
            check(cudaMemcpyAsync(h_atm_counts_, d_off_ + n, sizeof(long long), cudaMemcpyDeviceToHost, stream), "total");
            check(cudaMemcpyAsync(h_atm_counts_ + 1, d_maxcnt_, sizeof(int), cudaMemcpyDeviceToHost, stream), "max");
            check(cudaStreamSynchronize(stream), "neighbour count");
            const long long total = h_atm_counts_[0];
            const int maxcnt = (int)(reinterpret_cast<int*>(h_atm_counts_ + 1)[0]);
            last_triples_entries_ = total;
            if (total > nbr_cap_) {
                void* pj = d_nbr_j_; void* pgd = d_nbr_gend_; void* pv = d_nbr_v_;
                free_block(pj); free_block(pgd); free_block(pv);
                nbr_cap_ = total + total / 4 + 1024;
                d_nbr_j_ = dev_alloc<int>(nbr_cap_);
                d_nbr_gend_ = dev_alloc<int>(nbr_cap_);
                d_nbr_v_ = dev_alloc<double4>(nbr_cap_);
            }
            // a captured sequence keeps the list length it was captured with: reserve headroom
            stride = std::max(maxcnt, 1);
            if (graph_on_) {
                if (maxcnt > atm_stride_) atm_stride_ = maxcnt + maxcnt / 4 + 32;
                stride = atm_stride_;
            }
            // the slot buffers are sized for the largest resident grid (one block per SM and unit of occupancy)
            const long long grid = (long long)sms_ * std::max(atm_occupancy(c.mixed, true), atm_occupancy(c.mixed, false));
            const long long need = grid * stride * 8;   // per-entry accumulators (up to 8 doubles)
            if (need > slot_cap_) {
                void* p = d_slot_acc_;
                free_block(p);
                slot_cap_ = need + need / 4;
                d_slot_acc_ = dev_alloc<double>(slot_cap_);
            }
            const long long scr_need = grid * stride * (long long)atm_slot_bytes(false);
            if (scr_need > slot_scr_cap_) {
                void* p = d_slot_scr_;
                free_block(p);
                slot_scr_cap_ = scr_need + scr_need / 4;
                d_slot_scr_ = dev_alloc<unsigned char>(slot_scr_cap_);
            }
        }
        launch_atm_guard(d_off_ + n, d_maxcnt_, nbr_cap_, stride, d_guard_, stream);
        launch_nbr_fill(b, c, d_sys_mol_, d_off_, d_cnt_, d_nbr_j_, d_nbr_gend_, d_nbr_v_, d_guard_, stream);
        check(cudaMemsetAsync(d_queue_, 0, sizeof(unsigned int), stream), "memset");
        w.atm_guard = d_guard_;
        if (profiling_ && !capturing_) check(cudaEventRecord(kev_[2], stream), "cudaEventRecord");
        if (c.grad) check(cudaMemsetAsync(d_fxacc_, 0, sizeof(unsigned long long) * 8 * n, stream), "memset");
        launch_triples(b, s, d, c, part_, w, d_c6mat_, d_c6mat_off_, d_off_, d_cnt_, d_nbr_j_, d_nbr_gend_, d_nbr_v_,
                       d_queue_, d_slot_acc_, d_slot_scr_, stride, blocks, any_periodic_, d_e3_, d_sig3_, d_fxacc_,
                       stream);
        if (c.grad) launch_atm_fixed(n, d_fxacc_, d_guard_, w, stream);
    }
    if (!mol_order_.empty()) {
        // after the root kernel, which writes zeros for the molecules' atoms
        if (profiling_ && !capturing_ && root_atoms_ == 0) check(cudaEventRecord(kev_[2], stream), "cudaEventRecord");
        const int nmol = (int)mol_order_.size();
        const int mblocks = std::max(1, std::min(nmol, sms_ * atm_mol_occupancy(c.mixed, c.grad)));
        check(cudaMemsetAsync(d_queue_ + 1, 0, sizeof(unsigned int), stream), "memset");
        launch_triples_mol(b, s, d, c, part_, w, d_c6mat_, d_c6mat_off_, d_mol_order_, nmol, d_queue_ + 1, mblocks,
                           d_e3_, d_sig3_, stream);
    }
    if (profiling_ && !capturing_) {
        check(cudaEventRecord(kev_[3], stream), "cudaEventRecord");
        kev3_recorded_ = true;
    }
    w.e3_atom = d_e3_;
    w.sig3_atom = c.grad ? d_sig3_ : nullptr;
}

void Engine::stage_times(double out[kTimes])
{
    for (int k = 0; k < kTimes; k++) out[k] = 0.0;
    if (!ev_recorded_) return;
    check(cudaEventSynchronize(ev_[kStages]), "cudaEventSynchronize");
    for (int k = 0; k < kStages; k++) {
        float ms = 0.f;
        check(cudaEventElapsedTime(&ms, ev_[k], ev_[k + 1]), "cudaEventElapsedTime");
        out[k] = ms;
    }
    float ms = 0.f;
    if (out[3] > 0.0 && cudaEventElapsedTime(&ms, kev_[0], kev_[1]) == cudaSuccess) out[kStages] = ms;
    (void)cudaGetLastError();
    if (kev3_recorded_ && cudaEventElapsedTime(&ms, kev_[2], kev_[3]) == cudaSuccess) out[kStages + 1] = ms;
    (void)cudaGetLastError();
}

int Engine::atm_occupancy(bool mixed, bool grad)
{
    int& occ = atm_occ_[mixed ? 1 : 0][grad ? 1 : 0];
    if (occ == 0) occ = atm_blocks_per_sm(mixed, grad);
    return occ;
}

int Engine::atm_mol_occupancy(bool mixed, bool grad)
{
    int& occ = atm_mol_occ_[mixed ? 1 : 0][grad ? 1 : 0];
    if (occ == 0) occ = atm_mol_blocks_per_sm(mixed, grad);
    return occ;
}

int Engine::atm_blocks(bool mixed, bool grad)
{
    const int occ = atm_occupancy(mixed, grad);
    return tune_.atm_blocks_per_sm > 0 ? std::min(tune_.atm_blocks_per_sm, occ) : occ;
}

// ------------------------------------------------------------------ graph --

void Engine::drop_graph()
{
    if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
    graph_exec_ = nullptr;
    graph_valid_ = false;
}

void Engine::reduce(double* buffer, int count, cudaStream_t stream)
{
    check(cudaGetLastError(), "kernel launch");
    if (reducer_(buffer, count, stream, reducer_user_) != 0) throw Error("The reducer reported an error");
}

void Engine::set_reducer(Reducer fn, void* user, int part, int nparts)
{
    check(cudaSetDevice(device_), "cudaSetDevice");
    if (fn && graph_on_) throw Error("A reducer cannot be combined with the captured launch sequence");
    if (fn && (nparts < 1 || part < 0 || part >= nparts)) throw Error("Invalid dispersion work partition");
    reducer_ = fn;
    reducer_user_ = user;
    if (fn) {
        if (!d_red_) {
            const size_t len = (size_t)nsys_ * (1 + kParamGrad + 9) + 3 * (size_t)natoms_;
            d_red_ = dev_alloc<double>(len);
            check(cudaMemsetAsync(d_red_, 0, sizeof(double) * len, stream_), "memset");
            check(cudaStreamSynchronize(stream_), "memset");
        }
        set_partition(part, nparts, true);
    } else {
        set_partition(0, 1, false);
    }
}

void Engine::set_graph(bool on)
{
    check(cudaSetDevice(device_), "cudaSetDevice");
    if (on && reducer_) throw Error("A reducer cannot be combined with the captured launch sequence");
    if (!on) drop_graph();
    graph_on_ = on;
}

void Engine::set_tuning(const Tuning& t)
{
    if (t.pair_split != 0 && t.pair_split != 1 && t.pair_split != 2 && t.pair_split != 4)
        throw Error("Work items per tile pair must be 1, 2 or 4 (0 chooses)");
    if (!(t.morton_cell >= 0.0) || !std::isfinite(t.morton_cell))
        throw Error("Sort cell must be positive (Morton order) or 0 (column order)");
    if (t.atm_blocks_per_sm < 0) throw Error("Three-body blocks per SM must not be negative");
    if (t.atm_mol < 0 || t.atm_mol > 2) throw Error("Molecule kernel mode must be 0, 1 or 2");
    check(cudaSetDevice(device_), "cudaSetDevice");
    const bool remol = t.atm_mol != tune_.atm_mol;
    tune_ = t;
    if (remol) configure_molecules();
    graph_valid_ = false;
}

Engine::GraphKey Engine::make_key(const Damp& d, bool grad, bool pg) const
{
    GraphKey k;
    std::memset(&k, 0, sizeof(k));   // the key is compared bytewise
    k.damp = d;
    k.cut = cut_;
    k.part = part_;
    k.tune = tune_;
    k.grad = grad; k.pg = pg; k.counting = counting_; k.mixed = mixed_; k.cn_part = cn_partitioned_;
    return k;
}

void Engine::capture(const Damp& d, const GraphKey& key, bool grad, bool pg)
{
    cudaGraph_t g = nullptr;
    capturing_ = true;
    check(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
    try {
        run(d, d_pos_in_, d_energies_, grad ? d_grad_out_ : nullptr, grad ? d_sigma_ : nullptr,
            pg ? d_pg_out_ : nullptr, grad, stream_);
    } catch (...) {
        cudaStreamEndCapture(stream_, &g);
        if (g) cudaGraphDestroy(g);
        capturing_ = false;
        throw;
    }
    capturing_ = false;
    check(cudaStreamEndCapture(stream_, &g), "cudaStreamEndCapture");
    // kernels one replay launches: the kernel nodes of the captured graph
    {
        size_t nn = 0;
        graph_kernels_ = 0;
        if (cudaGraphGetNodes(g, nullptr, &nn) == cudaSuccess && nn > 0) {
            std::vector<cudaGraphNode_t> nodes(nn);
            if (cudaGraphGetNodes(g, nodes.data(), &nn) == cudaSuccess)
                for (size_t k = 0; k < nn; k++) {
                    cudaGraphNodeType t;
                    if (cudaGraphNodeGetType(nodes[k], &t) == cudaSuccess && t == cudaGraphNodeTypeKernel)
                        graph_kernels_++;
                }
        }
    }
    bool updated = false;
    if (graph_exec_) {
        cudaGraphExecUpdateResultInfo info;
        updated = cudaGraphExecUpdate(graph_exec_, g, &info) == cudaSuccess;
        if (!updated) {
            (void)cudaGetLastError();
            drop_graph();
        }
    }
    if (!updated) {
        const cudaError_t e = cudaGraphInstantiate(&graph_exec_, g, 0);
        cudaGraphDestroy(g);
        check(e, "cudaGraphInstantiate");
    } else {
        cudaGraphDestroy(g);
    }
    graph_key_ = key;
    graph_epoch_ = alloc_epoch_;
    graph_valid_ = true;
}

void Engine::run_graphed(const Damp& d, bool grad, bool pg, cudaStream_t stream)
{
    if (pg && !damping_has_param_grad(d.kind))
        throw Error("Damping parameter derivatives are available for the rational and zero damping only");
    ensure_images(stream);
    ensure_workspace(grad, pg, false);
    upload_pair_table(d, stream);
    const GraphKey key = make_key(d, grad, pg);
    const bool threebody = std::fabs(d.s9) >= DBL_EPSILON || pg;
    if (graph_valid_ && graph_epoch_ == alloc_epoch_ && std::memcmp(&key, &graph_key_, sizeof(key)) == 0) {
        check(cudaGraphLaunch(graph_exec_, stream), "cudaGraphLaunch");
        if (!threebody) return;
        // the three-body lists must have fitted the buffers the graph was captured with
        check(cudaMemcpyAsync(h_guard_, d_guard_, sizeof(int), cudaMemcpyDeviceToHost, stream), "guard");
        check(cudaStreamSynchronize(stream), "graph");
        if (*h_guard_ == 0) return;
        graph_valid_ = false;
    }
    // ordinary evaluation: this call's results, and the list sizes for the capture
    run(d, d_pos_in_, d_energies_, grad ? d_grad_out_ : nullptr, grad ? d_sigma_ : nullptr, pg ? d_pg_out_ : nullptr,
        grad, stream);
    // the capture records work on the engine stream; it must not overlap buffers still in use
    check(cudaStreamSynchronize(stream), "evaluation");
    capture(d, key, grad, pg);
}

double* Engine::input_buffer()
{
    check(cudaSetDevice(device_), "cudaSetDevice");
    ensure_workspace(true, false, false);
    return d_pos_in_;
}

double Engine::autotune(const Damp& d, const double* d_positions, bool grad, cudaStream_t stream)
{
    check(cudaSetDevice(device_), "cudaSetDevice");
    ensure_workspace(grad, false, false);
    const bool threebody = std::fabs(d.s9) >= DBL_EPSILON;
    cudaEvent_t e0, e1;
    check(cudaEventCreate(&e0), "cudaEventCreate");
    check(cudaEventCreate(&e1), "cudaEventCreate");
    const bool prof = profiling_;
    profiling_ = false;
    auto time_once = [&]() {
        // one run to size the buffers of this shape, then the faster of two timed runs
        double best = 1e30;
        for (int rep = 0; rep < 3; rep++) {
            check(cudaEventRecord(e0, stream), "cudaEventRecord");
            run(d, d_positions, d_energies_, grad ? d_grad_out_ : nullptr, grad ? d_sigma_ : nullptr, nullptr, grad,
                stream);
            check(cudaEventRecord(e1, stream), "cudaEventRecord");
            check(cudaEventSynchronize(e1), "cudaEventSynchronize");
            float ms = 0.f;
            check(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime");
            if (rep > 0) best = std::min(best, (double)ms);
        }
        return best;
    };
    Tuning best = tune_;
    double best_ms = 0.0;
    try {
        best_ms = time_once();
        auto consider = [&](Tuning t) {
            tune_ = t;
            const double ms = time_once();
            if (ms < best_ms) { best_ms = ms; best = t; }
            tune_ = best;
        };
        for (double cell : {0.0, 2.0, 3.0, 4.5, 6.0})
            if (cell != best.morton_cell) { Tuning t = best; t.morton_cell = cell; consider(t); }
        for (int sp : {1, 2, 4})
            if (sp != best.pair_split) { Tuning t = best; t.pair_split = sp; consider(t); }
        if (threebody) {
            // molecules: one block each, or the neighbour-list kernel
            bool any_mol = false;
            for (int sy = 0; sy < nsys_; sy++)
                any_mol = any_mol || (!(per_[3 * sy] || per_[3 * sy + 1] || per_[3 * sy + 2]) &&
                                      sys_natoms_[sy] <= atm_mol_max_atoms());
            if (any_mol)
                for (int mode : {1, 2})
                    if (mode != best.atm_mol) {
                        Tuning t = best; t.atm_mol = mode;
                        const bool remol = t.atm_mol != tune_.atm_mol;
                        tune_ = t;
                        if (remol) configure_molecules();
                        const double ms = time_once();
                        if (ms < best_ms) { best_ms = ms; best = t; }
                        tune_ = best;
                        configure_molecules();
                    }
            const int occ = atm_occupancy(mixed_, grad);
            const int cur = best.atm_blocks_per_sm > 0 ? std::min(best.atm_blocks_per_sm, occ) : occ;
            for (int bps = 1; bps <= occ; bps++)
                if (bps != cur) { Tuning t = best; t.atm_blocks_per_sm = bps; consider(t); }
        }
    } catch (...) {
        tune_ = best;
        configure_molecules();
        profiling_ = prof;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        throw;
    }
    tune_ = best;
    configure_molecules();
    profiling_ = prof;
    graph_valid_ = false;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return best_ms;
}

void Engine::evaluate_host(const Damp& d, const double* positions, double* energies, double* gradient,
                           double* sigma9)
{
    check(cudaSetDevice(device_), "cudaSetDevice");
    const bool grad = gradient != nullptr || sigma9 != nullptr;
    ensure_workspace(grad, false, false);
    const size_t nin = 3 * (size_t)natoms_;
    const size_t nout = nsys_ + 3 * (size_t)natoms_ + 9 * (size_t)nsys_;
    if (h_stage_len_ < nin + nout) {
        if (h_stage_) cudaFreeHost(h_stage_);
        h_stage_len_ = nin + nout;
        check(cudaMallocHost(&h_stage_, sizeof(double) * h_stage_len_), "cudaMallocHost");
    }
    double* hin = h_stage_;
    double* he = h_stage_ + nin;
    double* hg = he + nsys_;
    double* hs = hg + 3 * (size_t)natoms_;
    std::memcpy(hin, positions, sizeof(double) * nin);
    check(cudaMemcpyAsync(d_pos_in_, hin, sizeof(double) * nin, cudaMemcpyHostToDevice, stream_), "positions");
    if (graph_on_) run_graphed(d, grad, false, stream_);
    else run(d, d_pos_in_, d_energies_, grad ? d_grad_out_ : nullptr, grad ? d_sigma_ : nullptr, nullptr, grad, stream_);
    // the staging layout [energies | gradient | virials] is the device one
    check(cudaMemcpyAsync(he, d_energies_, sizeof(double) * (grad ? nout : nsys_), cudaMemcpyDeviceToHost, stream_),
          "results");
    check(cudaStreamSynchronize(stream_), "evaluate");
    std::memcpy(energies, he, sizeof(double) * nsys_);
    if (gradient) std::memcpy(gradient, hg, sizeof(double) * 3 * natoms_);
    if (sigma9) std::memcpy(sigma9, hs, sizeof(double) * 9 * nsys_);
}

void Engine::evaluate_device(const Damp& d, const double* d_positions, double* d_energies,
                             double* d_gradient, double* d_sigma9, double* d_param_grad,
                             cudaStream_t stream)
{
    check(cudaSetDevice(device_), "cudaSetDevice");
    const bool grad = d_gradient != nullptr || d_sigma9 != nullptr;
    if (!graph_on_) {
        run(d, d_positions, d_energies, d_gradient, d_sigma9, d_param_grad, grad, stream);
        return;
    }
    // the graph reads and writes engine-owned buffers
    const bool pg = d_param_grad != nullptr;
    ensure_workspace(grad, pg, false);
    const size_t n3 = 3 * (size_t)natoms_;
    check(cudaMemcpyAsync(d_pos_in_, d_positions, sizeof(double) * n3, cudaMemcpyDeviceToDevice, stream), "positions");
    run_graphed(d, grad, pg, stream);
    check(cudaMemcpyAsync(d_energies, d_energies_, sizeof(double) * nsys_, cudaMemcpyDeviceToDevice, stream), "energies");
    if (d_gradient)
        check(cudaMemcpyAsync(d_gradient, d_grad_out_, sizeof(double) * n3, cudaMemcpyDeviceToDevice, stream), "gradient");
    if (d_sigma9)
        check(cudaMemcpyAsync(d_sigma9, d_sigma_, sizeof(double) * 9 * nsys_, cudaMemcpyDeviceToDevice, stream), "sigma");
    if (pg)
        check(cudaMemcpyAsync(d_param_grad, d_pg_out_, sizeof(double) * kParamGrad * nsys_, cudaMemcpyDeviceToDevice,
                              stream), "parameter derivatives");
}

}  // namespace d3
