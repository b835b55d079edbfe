// C ABI of the B200 D3 library: the reference's dftd3_* entry points
// (include/s-dftd3.h) and the batched/device extensions (dftd3_b200.h).
//
// Handles own host copies of their inputs; a model owns the GPU engine of its
// structure (device tables, workspace, stream), created on first evaluation.
// Errors follow the reference convention (api.f90): the error handle is the
// first argument, a NULL error handle makes a call return silently, and the
// messages of the reference are kept where the reference has one.
#include <cfloat>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/dftd3_b200.h"
#include "d3_engine.h"
#include "d3_params.h"
#include "d3_tables.h"

namespace d3 {
bool noalloc_dispersion(const Damp& damp, int natoms, const int* numbers, const double* d_positions,
                        const double* lattice, const bool* periodic, const double* cutoffs, int precision,
                        double* d_energy, double* d_gradient, double* d_sigma, cudaStream_t stream, char* msg);
}

struct _dftd3_error {
    bool set = false;
    std::string message;
};

struct _dftd3_structure {
    int nat = 0;
    std::vector<int> numbers;
    std::vector<double> xyz;
    double lattice[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    bool periodic[3] = {false, false, false};
};

struct _dftd3_model {
    std::vector<int> numbers;
    bool has_cutoff = false;
    d3::Cutoffs cutoff;
    std::vector<uint8_t> ghost;
    int part = 0, nparts = 1;
    int precision = DFTD3_B200_PRECISION_FP64;
    bool has_tuning = false;
    d3::Tuning tuning;
    bool graph = false;
    std::unique_ptr<d3::Engine> engine;
};

struct _dftd3_param {
    bool supported = true;
    d3::Damp damp;
};

struct _dftd3_gcp {
    int unused = 0;
};

struct _dftd3_b200_batch {
    std::unique_ptr<d3::Engine> engine;
    std::vector<double> wrapped;
};

namespace {

void fail(dftd3_error err, const std::string& msg)
{
    if (!err) return;
    err->set = true;
    err->message = msg;
}

void unsupported(dftd3_error err, const char* what)
{
    fail(err, std::string(what) + " is not supported by the B200 DFT-D3 library");
}

bool finite_all(const double* v, size_t n)
{
    for (size_t k = 0; k < n; k++)
        if (!std::isfinite(v[k])) return false;
    return true;
}

template <class F>
void guarded(dftd3_error err, F&& f)
{
    try {
        f();
    } catch (const std::exception& e) {
        fail(err, e.what());
    }
}

}  // namespace

namespace {

// Launch shapes from the C array of dftd3_b200_set_*_tuning.
d3::Tuning tuning_from(const double* tuning)
{
    d3::Tuning t;
    t.morton_cell = tuning[0];
    t.pair_split = (int)tuning[1];
    t.atm_blocks_per_sm = (int)tuning[2];
    t.atm_mol = (int)tuning[3];
    if ((double)t.pair_split != tuning[1] || (double)t.atm_blocks_per_sm != tuning[2] || (double)t.atm_mol != tuning[3])
        throw d3::Error("Launch shape counts must be integers");
    return t;
}

// Method id of a method name as get_method_id does it (param.f90:96-114):
// '-' removed, letters outside quotes in lower case, trailing blanks ignored.
int method_id(const char* method)
{
    std::string lc;
    for (const char* c = method; *c; c++)
        if (*c != '-') lc.push_back(*c);
    bool quoted = false;
    char quote = 0;
    for (char& c : lc) {
        if (!quoted && (c == '"' || c == '\'')) { quoted = true; quote = c; continue; }
        if (quoted && c == quote) { quoted = false; continue; }
        if (!quoted && c >= 'A' && c <= 'Z') c = char(c - 'A' + 'a');
    }
    while (!lc.empty() && lc.back() == ' ') lc.pop_back();
    for (int k = 0; k < d3_n_method_aliases; k++)
        if (lc == d3_method_aliases[k].name) return d3_method_aliases[k].id;
    return 0;
}

// get_<family>_damping (param.f90:302-1326) and the load_*_damping entries
// (api.f90:588-1018): the record of the method, s9 = 1 when the three-body
// term is requested.
dftd3_param load_param(dftd3_error error, const char* method, bool atm, const d3_param_record* table, int n,
                       int kind)
{
    if (!error) return nullptr;
    if (!method) {
        fail(error, "Method name is missing");
        return nullptr;
    }
    const int id = method_id(method);
    const d3_param_record* rec = nullptr;
    for (int k = 0; id && k < n && !rec; k++)
        if (table[k].id == id) rec = &table[k];
    if (!rec) {
        fail(error, std::string("No entry for '") + method + "' present");
        return nullptr;
    }
    auto* p = new _dftd3_param();
    p->damp.kind = kind;
    p->damp.s6 = rec->v[0]; p->damp.s8 = rec->v[1]; p->damp.s9 = atm ? 1.0 : rec->v[2];
    p->damp.rs6 = rec->v[3]; p->damp.rs8 = rec->v[4];
    p->damp.a1 = rec->v[5]; p->damp.a2 = rec->v[6]; p->damp.alp = rec->v[7]; p->damp.bet = rec->v[8];
    return p;
}

}  // namespace

extern "C" {

int dftd3_get_version() { return 10000 * 1 + 100 * 6 + 0; }

bool dftd3_has_feature(char* feature)
{
    (void)feature;
    return false;
}

dftd3_error dftd3_new_error() { return new _dftd3_error(); }

int dftd3_check_error(dftd3_error error)
{
    if (!error) return 2;
    return error->set ? 1 : 0;
}

void dftd3_get_error(dftd3_error error, char* buffer, const int* buffersize)
{
    if (!error || !buffer || !error->set) return;
    // like f_c_character: copy at most size-1 characters and terminate
    size_t max_length = buffersize ? (size_t)(*buffersize > 0 ? *buffersize : 0) : error->message.size() + 1;
    if (max_length == 0) return;
    const size_t n = std::min(error->message.size(), max_length - 1);
    std::memcpy(buffer, error->message.data(), n);
    buffer[n] = '\0';
}

void dftd3_delete_error(dftd3_error* error)
{
    if (error && *error) {
        delete *error;
        *error = nullptr;
    }
}

dftd3_structure dftd3_new_structure(dftd3_error error, const int natoms, const int* numbers,
                                    const double* positions, const double* lattice, const bool* periodic)
{
    if (!error) return nullptr;
    if (natoms < 0 || (natoms > 0 && (!numbers || !positions))) {
        fail(error, "Invalid molecular structure data provided");
        return nullptr;
    }
    auto* mol = new _dftd3_structure();
    mol->nat = natoms;
    mol->numbers.assign(numbers, numbers + natoms);
    mol->xyz.assign(positions, positions + 3 * (size_t)natoms);
    if (lattice) std::memcpy(mol->lattice, lattice, sizeof(mol->lattice));
    for (int k = 0; k < 3; k++) mol->periodic[k] = periodic ? periodic[k] : (lattice != nullptr);
    d3::wrap_to_central_cell(natoms, mol->xyz.data(), mol->lattice, mol->periodic);
    if (d3::has_overlapping_atoms(natoms, mol->xyz.data())) fail(error, "Too close interatomic distances found");
    return mol;
}

void dftd3_delete_structure(dftd3_structure* mol)
{
    if (mol && *mol) {
        delete *mol;
        *mol = nullptr;
    }
}

void dftd3_update_structure(dftd3_error error, dftd3_structure mol, const double* positions, const double* lattice)
{
    if (!error) return;
    if (!mol) {
        fail(error, "Molecular structure data is missing");
        return;
    }
    if (mol->nat <= 0 || !positions) {
        fail(error, "Invalid molecular structure data provided");
        return;
    }
    std::memcpy(mol->xyz.data(), positions, sizeof(double) * 3 * mol->nat);
    if (lattice) std::memcpy(mol->lattice, lattice, sizeof(mol->lattice));
    d3::wrap_to_central_cell(mol->nat, mol->xyz.data(), mol->lattice, mol->periodic);
    if (d3::has_overlapping_atoms(mol->nat, mol->xyz.data())) fail(error, "Too close interatomic distances found");
}

dftd3_model dftd3_new_d3_model(dftd3_error error, dftd3_structure mol)
{
    if (!error) return nullptr;
    if (!mol) {
        fail(error, "Molecular structure data is missing");
        return nullptr;
    }
    for (int z : mol->numbers)
        if (z < 1 || z > D3_MAX_ELEM) {
            fail(error, "Unsupported element with atomic number " + std::to_string(z));
            return nullptr;
        }
    auto* disp = new _dftd3_model();
    disp->numbers = mol->numbers;
    disp->ghost.assign(mol->nat, 0);
    return disp;
}

void dftd3_set_model_realspace_cutoff(dftd3_error error, dftd3_model model, double disp2, double disp3, double cn)
{
    if (!error) return;
    if (!model) {
        fail(error, "D3 dispersion model is missing");
        return;
    }
    model->has_cutoff = true;
    model->cutoff = d3::Cutoffs{disp2, disp3, cn, 0.0, 0.0};
    if (model->engine) model->engine->set_cutoffs(model->cutoff);
}

void dftd3_set_model_realspace_cutoff_smooth(dftd3_error error, dftd3_model model, double disp2, double disp3,
                                             double cn, double width2, double width3)
{
    if (!error) return;
    if (!model) {
        fail(error, "D3 dispersion model is missing");
        return;
    }
    model->has_cutoff = true;
    model->cutoff = d3::Cutoffs{disp2, disp3, cn, width2, width3};
    if (model->engine) model->engine->set_cutoffs(model->cutoff);
}

void dftd3_set_model_ghost_index(dftd3_error error, dftd3_model model, const int* ghost, int nidx)
{
    if (!error) return;
    if (!model) {
        fail(error, "D3 dispersion model is missing");
        return;
    }
    for (int k = 0; k < nidx; k++) {
        const int iat = ghost[k];
        if (iat >= 0 && iat < (int)model->ghost.size()) model->ghost[iat] = 1;
        else fail(error, "Index out of bounds");
    }
    if (model->engine) guarded(error, [&] { model->engine->set_ghost(model->ghost); });
}

void dftd3_set_model_ewald(dftd3_error error, dftd3_model model, int, double, double, int)
{
    if (!error) return;
    if (!model) {
        fail(error, "D3 dispersion model is missing");
        return;
    }
    unsupported(error, "Ewald summation");
}

void dftd3_set_model_work_partition(dftd3_error error, dftd3_model model, int part, int nparts)
{
    if (!error) return;
    if (!model) {
        fail(error, "D3 dispersion model is missing");
        return;
    }
    // new_work_partition, partition.f90:80-100
    if (nparts <= 0 || part < 0 || part >= nparts) {
        fail(error, "Invalid dispersion work partition");
        return;
    }
    model->part = part;
    model->nparts = nparts;
    if (model->engine) model->engine->set_partition(part, nparts, false);
}

void dftd3_set_model_mpi_comm(dftd3_error error, dftd3_model model, int)
{
    if (!error) return;
    if (!model) {
        fail(error, "D3 dispersion model is missing");
        return;
    }
    fail(error, "s-dftd3 was built without MPI support");
}

void dftd3_delete_model(dftd3_model* disp)
{
    if (disp && *disp) {
        delete *disp;
        *disp = nullptr;
    }
}

dftd3_param dftd3_new_zero_damping(dftd3_error error, double s6, double s8, double s9, double rs6, double rs8,
                                   double alp)
{
    if (!error) return nullptr;
    auto* p = new _dftd3_param();
    p->damp.kind = d3::kZero;
    p->damp.s6 = s6; p->damp.s8 = s8; p->damp.s9 = s9;
    p->damp.rs6 = rs6; p->damp.rs8 = rs8; p->damp.alp = alp;
    return p;
}

dftd3_param dftd3_new_rational_damping(dftd3_error error, double s6, double s8, double s9, double a1, double a2,
                                       double alp)
{
    if (!error) return nullptr;
    auto* p = new _dftd3_param();
    p->damp.kind = d3::kRational;
    p->damp.s6 = s6; p->damp.s8 = s8; p->damp.s9 = s9;
    p->damp.a1 = a1; p->damp.a2 = a2; p->damp.alp = alp;
    return p;
}

dftd3_param dftd3_load_zero_damping(dftd3_error error, char* method, bool atm)
{
    return load_param(error, method, atm, d3_zero_params, d3_n_zero_params, d3::kZero);
}

dftd3_param dftd3_load_rational_damping(dftd3_error error, char* method, bool atm)
{
    return load_param(error, method, atm, d3_rational_params, d3_n_rational_params, d3::kRational);
}

dftd3_param dftd3_load_mrational_damping(dftd3_error error, char* method, bool atm)
{
    // the modified rational records are evaluated with the rational damping
    // function (api.f90:710-745 constructs a rational_damping_param)
    return load_param(error, method, atm, d3_mrational_params, d3_n_mrational_params, d3::kRational);
}

dftd3_param dftd3_load_mzero_damping(dftd3_error error, char* method, bool atm)
{
    return load_param(error, method, atm, d3_mzero_params, d3_n_mzero_params, d3::kMZero);
}

dftd3_param dftd3_load_optimizedpower_damping(dftd3_error error, char* method, bool atm)
{
    return load_param(error, method, atm, d3_optimizedpower_params, d3_n_optimizedpower_params,
                      d3::kOptimizedPower);
}

dftd3_param dftd3_load_cso_damping(dftd3_error error, char* method, bool atm)
{
    return load_param(error, method, atm, d3_cso_params, d3_n_cso_params, d3::kCSO);
}

dftd3_param dftd3_load_z_damping(dftd3_error error, char* method, bool atm)
{
    // get_z_damping has no records (param.f90:1297-1326): every name fails
    return load_param(error, method, atm, d3_z_params, d3_n_z_params, d3::kZDamping);
}

dftd3_param dftd3_new_mzero_damping(dftd3_error error, double s6, double s8, double s9, double rs6, double rs8,
                                    double alp, double bet)
{
    // new_mzero_damping_api, api.f90:748-777
    if (!error) return nullptr;
    auto* p = new _dftd3_param();
    p->damp.kind = d3::kMZero;
    p->damp.s6 = s6; p->damp.s8 = s8; p->damp.s9 = s9;
    p->damp.rs6 = rs6; p->damp.rs8 = rs8; p->damp.alp = alp; p->damp.bet = bet;
    return p;
}

dftd3_param dftd3_new_mrational_damping(dftd3_error error, double s6, double s8, double s9, double a1, double a2,
                                        double alp)
{
    // the modified rational form evaluates the rational damping function with
    // other parameters (rational.f90 serves both, api.f90:694-722)
    return dftd3_new_rational_damping(error, s6, s8, s9, a1, a2, alp);
}

dftd3_param dftd3_new_optimizedpower_damping(dftd3_error error, double s6, double s8, double s9, double a1,
                                             double a2, double alp, double bet)
{
    // new_optimizedpower_damping_api, api.f90:817-846
    if (!error) return nullptr;
    auto* p = new _dftd3_param();
    p->damp.kind = d3::kOptimizedPower;
    p->damp.s6 = s6; p->damp.s8 = s8; p->damp.s9 = s9;
    p->damp.a1 = a1; p->damp.a2 = a2; p->damp.alp = alp; p->damp.bet = bet;
    return p;
}

dftd3_param dftd3_new_cso_damping(dftd3_error error, double s6, double s9, double a1, double a2, double a3,
                                  double a4, double alp)
{
    // new_cso_damping_api, api.f90:886-915: a3 and a4 travel as rs6 and rs8
    if (!error) return nullptr;
    auto* p = new _dftd3_param();
    p->damp.kind = d3::kCSO;
    p->damp.s6 = s6; p->damp.s9 = s9;
    p->damp.a1 = a1; p->damp.a2 = a2; p->damp.rs6 = a3; p->damp.rs8 = a4; p->damp.alp = alp;
    return p;
}

dftd3_param dftd3_new_z_damping(dftd3_error error, double s6, double s8, double s9, double a1, double alp)
{
    // new_z_damping_api, api.f90:955-982 (a2 = 0)
    if (!error) return nullptr;
    auto* p = new _dftd3_param();
    p->damp.kind = d3::kZDamping;
    p->damp.s6 = s6; p->damp.s8 = s8; p->damp.s9 = s9;
    p->damp.a1 = a1; p->damp.a2 = 0.0; p->damp.alp = alp;
    return p;
}

void dftd3_delete_param(dftd3_param* param)
{
    if (param && *param) {
        delete *param;
        *param = nullptr;
    }
}

dftd3_gcp dftd3_load_gcp_param(dftd3_error error, dftd3_structure, char*, char*)
{
    if (!error) return nullptr;
    unsupported(error, "The geometric counter-poise correction");
    return nullptr;
}

void dftd3_set_gcp_realspace_cutoff(dftd3_error error, dftd3_gcp, double, double)
{
    if (error) unsupported(error, "The geometric counter-poise correction");
}

void dftd3_set_gcp_work_partition(dftd3_error error, dftd3_gcp, int, int)
{
    if (error) unsupported(error, "The geometric counter-poise correction");
}

void dftd3_set_gcp_mpi_comm(dftd3_error error, dftd3_gcp, int)
{
    if (error) unsupported(error, "The geometric counter-poise correction");
}

void dftd3_delete_gcp(dftd3_gcp* gcp)
{
    if (gcp && *gcp) {
        delete *gcp;
        *gcp = nullptr;
    }
}

// The model's engine, created on first use for the structure the model was
// built for, with the model's settings; the lattice follows the structure.
static void model_engine(dftd3_model disp, dftd3_structure mol)
{
    if (!disp->engine) {
        disp->engine = std::make_unique<d3::Engine>(1, &mol->nat, mol->numbers.data(), mol->lattice, mol->periodic);
        if (disp->has_cutoff) disp->engine->set_cutoffs(disp->cutoff);
        disp->engine->set_ghost(disp->ghost);
        disp->engine->set_partition(disp->part, disp->nparts, false);
        disp->engine->set_precision(disp->precision);
        if (disp->has_tuning) disp->engine->set_tuning(disp->tuning);
        if (disp->graph) disp->engine->set_graph(true);
    }
    disp->engine->set_lattices(mol->lattice);
}

void dftd3_get_dispersion(dftd3_error error, dftd3_structure mol, dftd3_model disp, dftd3_param param,
                          double* energy, double* gradient, double* sigma)
{
    // get_dispersion_api, api.f90:1038-1111
    if (!error) return;
    if (!mol) {
        fail(error, "Molecular structure data is missing");
        return;
    }
    if (!disp) {
        fail(error, "Dispersion model is missing");
        return;
    }
    if (!param) {
        fail(error, "Damping parameters are missing");
        return;
    }
    if (!param->supported) {
        fail(error, "Damping parameters are not initialized");
        return;
    }
    if (disp->numbers != mol->numbers) {
        fail(error, "Dispersion model does not match the molecular structure");
        return;
    }
    if (!finite_all(mol->xyz.data(), mol->xyz.size())) {
        fail(error, "Non-finite atomic positions");
        return;
    }
    guarded(error, [&] {
        model_engine(disp, mol);
        double e = 0.0;
        double s9[9];
        disp->engine->evaluate_host(param->damp, mol->xyz.data(), &e, gradient, sigma ? s9 : nullptr);
        if (energy) *energy = e;
        if (sigma) std::memcpy(sigma, s9, sizeof(s9));
    });
}

void dftd3_get_pairwise_dispersion(dftd3_error error, dftd3_structure mol, dftd3_model disp, dftd3_param param,
                                   double* pair_energy2, double* pair_energy3)
{
    // get_pairwise_dispersion_api, api.f90:1180-1236: both [nat][nat]
    // matrices are overwritten (symmetric, so either storage order reads them)
    if (!error) return;
    if (!mol) {
        fail(error, "Molecular structure data is missing");
        return;
    }
    if (!disp) {
        fail(error, "Dispersion model is missing");
        return;
    }
    if (!param) {
        fail(error, "Damping parameters are missing");
        return;
    }
    if (!param->supported) {
        fail(error, "Damping parameters are not initialized");
        return;
    }
    if (!pair_energy2 || !pair_energy3) {
        fail(error, "Pairwise energy arrays are missing");
        return;
    }
    if (disp->numbers != mol->numbers) {
        fail(error, "Dispersion model does not match the molecular structure");
        return;
    }
    if (!finite_all(mol->xyz.data(), mol->xyz.size())) {
        fail(error, "Non-finite atomic positions");
        return;
    }
    guarded(error, [&] {
        model_engine(disp, mol);
        disp->engine->pairwise_host(param->damp, mol->xyz.data(), pair_energy2, pair_energy3);
    });
}

void dftd3_get_dispersion_hessian(dftd3_error error, dftd3_structure mol, dftd3_model disp, dftd3_param param,
                                  double* energy, double* hessian)
{
    // get_dispersion_hessian_api, api.f90:1115-1176: the energy and the
    // [3n][3n] Hessian (symmetric, so either storage order reads it)
    if (!error) return;
    if (!mol) {
        fail(error, "Molecular structure data is missing");
        return;
    }
    if (!disp) {
        fail(error, "Dispersion model is missing");
        return;
    }
    if (!param) {
        fail(error, "Damping parameters are missing");
        return;
    }
    if (!param->supported) {
        fail(error, "Damping parameters are not initialized");
        return;
    }
    if (!hessian) {
        fail(error, "Hessian array is missing");
        return;
    }
    if (disp->numbers != mol->numbers) {
        fail(error, "Dispersion model does not match the molecular structure");
        return;
    }
    if (!finite_all(mol->xyz.data(), mol->xyz.size())) {
        fail(error, "Non-finite atomic positions");
        return;
    }
    guarded(error, [&] {
        model_engine(disp, mol);
        double e = 0.0;
        disp->engine->evaluate_host(param->damp, mol->xyz.data(), &e, nullptr, nullptr);
        if (energy) *energy = e;
        disp->engine->hessian_host(param->damp, mol->xyz.data(), hessian);
    });
}

void dftd3_get_counterpoise(dftd3_error error, dftd3_structure, dftd3_gcp, double*, double*, double*)
{
    if (error) unsupported(error, "The geometric counter-poise correction");
}

void dftd3_get_counterpoise_hessian(dftd3_error error, dftd3_structure, dftd3_gcp, double*, double*)
{
    if (error) unsupported(error, "The geometric counter-poise correction");
}

// ------------------------------------------------------------- extensions --

void dftd3_b200_set_model_tuning(dftd3_error error, dftd3_model model, const double* tuning)
{
    if (!error) return;
    if (!model || !tuning) {
        fail(error, "D3 dispersion model is missing");
        return;
    }
    guarded(error, [&] {
        const d3::Tuning t = tuning_from(tuning);
        if (t.pair_split != 0 && t.pair_split != 1 && t.pair_split != 2 && t.pair_split != 4)
            throw d3::Error("Work items per tile pair must be 1, 2 or 4 (0 chooses)");
        model->tuning = t;
        model->has_tuning = true;
        if (model->engine) model->engine->set_tuning(t);
    });
}

void dftd3_b200_set_model_precision(dftd3_error error, dftd3_model model, int precision)
{
    if (!error) return;
    if (!model) {
        fail(error, "D3 dispersion model is missing");
        return;
    }
    if (precision != DFTD3_B200_PRECISION_FP64 && precision != DFTD3_B200_PRECISION_MIXED) {
        fail(error, "Invalid precision selector");
        return;
    }
    model->precision = precision;
    if (model->engine) model->engine->set_precision(precision);
}

void dftd3_b200_set_model_graph(dftd3_error error, dftd3_model model, int enable)
{
    if (!error) return;
    if (!model) {
        fail(error, "D3 dispersion model is missing");
        return;
    }
    model->graph = enable != 0;
    if (model->engine) guarded(error, [&] { model->engine->set_graph(model->graph); });
}

dftd3_b200_batch dftd3_b200_new_batch(dftd3_error error, int nsys, const int* natoms, const int* numbers,
                                      const double* lattices, const bool* periodic)
{
    if (!error) return nullptr;
    if (nsys <= 0 || !natoms || !numbers) {
        fail(error, "Invalid batch description");
        return nullptr;
    }
    dftd3_b200_batch b = nullptr;
    guarded(error, [&] {
        auto* nb = new _dftd3_b200_batch();
        try {
            nb->engine = std::make_unique<d3::Engine>(nsys, natoms, numbers, lattices, periodic);
        } catch (...) {
            delete nb;
            throw;
        }
        b = nb;
    });
    return b;
}

void dftd3_b200_set_batch_realspace_cutoff(dftd3_error error, dftd3_b200_batch batch, double disp2, double disp3,
                                           double cn, double width2, double width3)
{
    if (!error) return;
    if (!batch) {
        fail(error, "Batch is missing");
        return;
    }
    batch->engine->set_cutoffs(d3::Cutoffs{disp2, disp3, cn, width2, width3});
}

void dftd3_b200_set_batch_precision(dftd3_error error, dftd3_b200_batch batch, int precision)
{
    if (!error) return;
    if (!batch) {
        fail(error, "Batch is missing");
        return;
    }
    if (precision != DFTD3_B200_PRECISION_FP64 && precision != DFTD3_B200_PRECISION_MIXED) {
        fail(error, "Invalid precision selector");
        return;
    }
    batch->engine->set_precision(precision);
}

void dftd3_b200_get_dispersion_batched(dftd3_error error, dftd3_b200_batch batch, dftd3_param param,
                                       const double* positions, const double* lattices, double* energies,
                                       double* gradient, double* sigma)
{
    if (!error) return;
    if (!batch) {
        fail(error, "Batch is missing");
        return;
    }
    if (!param) {
        fail(error, "Damping parameters are missing");
        return;
    }
    if (!positions || !energies) {
        fail(error, "Invalid batch buffers");
        return;
    }
    guarded(error, [&] {
        d3::Engine& eng = *batch->engine;
        eng.set_lattices(lattices);
        const int n = eng.natoms();
        batch->wrapped.assign(positions, positions + 3 * (size_t)n);
        if (!finite_all(batch->wrapped.data(), batch->wrapped.size())) throw d3::Error("Non-finite atomic positions");
        for (int s = 0; s < eng.nsys(); s++) {
            const int a0 = eng.atom_off()[s], a1 = eng.atom_off()[s + 1];
            d3::wrap_to_central_cell(a1 - a0, batch->wrapped.data() + 3 * a0, eng.lattice(s), eng.periodic(s));
        }
        eng.evaluate_host(param->damp, batch->wrapped.data(), energies, gradient, sigma);
    });
}

void dftd3_b200_get_dispersion_device(dftd3_error error, dftd3_b200_batch batch, dftd3_param param,
                                      const double* d_positions, const double* lattices, double* d_energies,
                                      double* d_gradient, double* d_sigma, double* d_param_grad, void* stream)
{
    if (!error) return;
    if (!batch) {
        fail(error, "Batch is missing");
        return;
    }
    if (!param) {
        fail(error, "Damping parameters are missing");
        return;
    }
    if (!d_positions || !d_energies) {
        fail(error, "Invalid batch buffers");
        return;
    }
    guarded(error, [&] {
        batch->engine->set_lattices(lattices);
        batch->engine->evaluate_device(param->damp, d_positions, d_energies, d_gradient, d_sigma, d_param_grad,
                                       static_cast<cudaStream_t>(stream));
    });
}

void dftd3_b200_set_batch_counting(dftd3_error error, dftd3_b200_batch batch, int enable)
{
    if (!error) return;
    if (!batch) {
        fail(error, "Batch is missing");
        return;
    }
    batch->engine->set_counting(enable != 0);
}

void dftd3_b200_get_batch_counts(dftd3_error error, dftd3_b200_batch batch, long long* counts)
{
    if (!error) return;
    if (!batch || !counts) {
        fail(error, "Batch is missing");
        return;
    }
    guarded(error, [&] { batch->engine->counts(counts); });
}

void dftd3_b200_set_batch_profiling(dftd3_error error, dftd3_b200_batch batch, int enable)
{
    if (!error) return;
    if (!batch) {
        fail(error, "Batch is missing");
        return;
    }
    batch->engine->set_profiling(enable != 0);
}

void dftd3_b200_get_batch_stage_times(dftd3_error error, dftd3_b200_batch batch, double* ms)
{
    if (!error) return;
    if (!batch || !ms) {
        fail(error, "Batch is missing");
        return;
    }
    guarded(error, [&] { batch->engine->stage_times(ms); });
}

void dftd3_b200_get_batch_graph_kernels(dftd3_error error, dftd3_b200_batch batch, long long* kernels)
{
    if (!error) return;
    if (!batch || !kernels) {
        fail(error, "Batch is missing");
        return;
    }
    *kernels = batch->engine->graph_kernels();
}

void dftd3_b200_get_dispersion_noalloc(dftd3_error error, dftd3_param param, int natoms, const int* numbers,
                                       const double* d_positions, const double* lattice, const bool* periodic,
                                       const double* cutoffs, int precision, double* d_energy,
                                       double* d_gradient, double* d_sigma, void* stream)
{
    if (!error) return;
    if (!param) {
        fail(error, "Damping parameters are missing");
        return;
    }
    char msg[256];
    if (!d3::noalloc_dispersion(param->damp, natoms, numbers, d_positions, lattice, periodic, cutoffs, precision,
                                d_energy, d_gradient, d_sigma, static_cast<cudaStream_t>(stream), msg))
        fail(error, msg);
}

void dftd3_b200_get_param_values(dftd3_error error, dftd3_param param, int* kind, double* values)
{
    if (!error) return;
    if (!param || !kind || !values) {
        fail(error, "Damping parameters are missing");
        return;
    }
    const d3::Damp& d = param->damp;
    *kind = d.kind;
    const double v[9] = {d.s6, d.s8, d.s9, d.a1, d.a2, d.rs6, d.rs8, d.alp, d.bet};
    for (int k = 0; k < 9; k++) values[k] = v[k];
}

double dftd3_b200_fma_peak(dftd3_error error, int precision)
{
    if (!error) return 0.0;
    double v = 0.0;
    guarded(error, [&] { v = d3::measure_fma_peak(precision == DFTD3_B200_PRECISION_FP64); });
    return v;
}

void dftd3_b200_set_batch_graph(dftd3_error error, dftd3_b200_batch batch, int enable)
{
    if (!error) return;
    if (!batch) {
        fail(error, "Batch is missing");
        return;
    }
    guarded(error, [&] { batch->engine->set_graph(enable != 0); });
}

void dftd3_b200_set_batch_tuning(dftd3_error error, dftd3_b200_batch batch, const double* tuning)
{
    if (!error) return;
    if (!batch || !tuning) {
        fail(error, "Batch is missing");
        return;
    }
    guarded(error, [&] {
        batch->engine->set_tuning(tuning_from(tuning));
    });
}

void dftd3_b200_get_batch_tuning(dftd3_error error, dftd3_b200_batch batch, double* tuning)
{
    if (!error) return;
    if (!batch || !tuning) {
        fail(error, "Batch is missing");
        return;
    }
    const d3::Tuning& t = batch->engine->tuning();
    tuning[0] = t.morton_cell;
    tuning[1] = t.pair_split;
    tuning[2] = t.atm_blocks_per_sm;
    tuning[3] = t.atm_mol;
}

double dftd3_b200_autotune_batch(dftd3_error error, dftd3_b200_batch batch, dftd3_param param,
                                 const double* positions, int gradient)
{
    if (!error) return 0.0;
    if (!batch) {
        fail(error, "Batch is missing");
        return 0.0;
    }
    if (!param) {
        fail(error, "Damping parameters are missing");
        return 0.0;
    }
    if (!positions) {
        fail(error, "Invalid batch buffers");
        return 0.0;
    }
    double ms = 0.0;
    guarded(error, [&] {
        d3::Engine& eng = *batch->engine;
        const int n = eng.natoms();
        batch->wrapped.assign(positions, positions + 3 * (size_t)n);
        if (!finite_all(batch->wrapped.data(), batch->wrapped.size())) throw d3::Error("Non-finite atomic positions");
        for (int s = 0; s < eng.nsys(); s++) {
            const int a0 = eng.atom_off()[s], a1 = eng.atom_off()[s + 1];
            d3::wrap_to_central_cell(a1 - a0, batch->wrapped.data() + 3 * a0, eng.lattice(s), eng.periodic(s));
        }
        double* d_pos = eng.input_buffer();
        cudaStream_t st = eng.stream();
        if (cudaMemcpyAsync(d_pos, batch->wrapped.data(), sizeof(double) * 3 * n, cudaMemcpyHostToDevice, st) !=
            cudaSuccess)
            throw d3::Error("CUDA error in autotune upload");
        ms = eng.autotune(param->damp, d_pos, gradient != 0, st);
    });
    return ms;
}

void dftd3_b200_set_batch_reducer(dftd3_error error, dftd3_b200_batch batch, dftd3_b200_reducer reducer, void* user,
                                  int part, int nparts)
{
    if (!error) return;
    if (!batch) {
        fail(error, "Batch is missing");
        return;
    }
    guarded(error, [&] { batch->engine->set_reducer(reducer, user, part, nparts); });
}

void dftd3_b200_delete_batch(dftd3_b200_batch* batch)
{
    if (batch && *batch) {
        delete *batch;
        *batch = nullptr;
    }
}

}  // extern "C"
