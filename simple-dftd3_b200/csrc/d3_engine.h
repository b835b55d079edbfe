// Host-side driver of the D3 pipeline: model tables, lattice images, device
// workspace and the launch sequence of one evaluation.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "d3_device.cuh"

#ifndef DIRECT_MAX_ATOMS
#define DIRECT_MAX_ATOMS 256
#endif
#ifndef DIRECT_MAX_TOTAL
#define DIRECT_MAX_TOTAL 2048
#endif

namespace d3 {

struct Cutoffs {
    // realspace_cutoff defaults (cutoff.f90:26-38)
    double disp2 = 60.0, disp3 = 40.0, cn = 40.0, width2 = 0.0, width3 = 0.0;
};

struct Error : std::runtime_error {
    using std::runtime_error::runtime_error;
};

// Lattice translations within rthr (get_lattice_points, cutoff.f90:140-227).
// lattice[3][3] holds one vector per row; periodic[3].
std::vector<double> lattice_points(const double* lattice, const bool* periodic, double rthr);

// Wrap positions into the central cell (wrap_to_central_cell, utils.f90:29-64).
void wrap_to_central_cell(int nat, double* xyz, const double* lattice, const bool* periodic);

// True if two atoms are closer than 1e-9 Bohr (verify_structure, api.f90:1517-1530).
bool has_overlapping_atoms(int nat, const double* xyz);

// Species set and the per-species D3 model tables (new_d3_model, model.f90:87-181).
struct ModelTables {
    std::vector<int> num;            // atomic number per species
    std::vector<double> rcov, r4r2, refcn, c6ref, rvdw;
    std::vector<float> c6ref_f;
    std::vector<int> nref;
    int nid() const { return (int)num.size(); }
};

class Engine {
public:
    // nsys systems with natoms[s] atoms each; numbers concatenated.
    // lattices[nsys][9] and periodic[nsys][3] may be null (molecules).
    Engine(int nsys, const int* natoms, const int* numbers, const double* lattices,
           const bool* periodic, int device = -1);
    ~Engine();
    Engine(const Engine&) = delete;
    Engine& operator=(const Engine&) = delete;

    int nsys() const { return nsys_; }
    int natoms() const { return natoms_; }
    const ModelTables& tables() const { return tab_; }
    const std::vector<int>& atom_off() const { return atom_off_; }
    bool periodic_any(int sys) const;
    const double* lattice(int sys) const { return &lat_[9 * sys]; }
    const bool* periodic(int sys) const { return &per_[3 * sys]; }

    void set_cutoffs(const Cutoffs& c) { cut_ = c; images_valid_ = false; }
    const Cutoffs& cutoffs() const { return cut_; }
    void set_ghost(const std::vector<uint8_t>& ghost);
    void set_partition(int part, int nparts, bool cn_partitioned);
    void set_precision(int mixed) { mixed_ = mixed != 0; }
    bool mixed() const { return mixed_; }
    void set_counting(bool on) { counting_ = on; }
    void counts(long long out[3]) const;
    // Replace the lattices (host, [nsys][9]); images are rebuilt lazily.
    void set_lattices(const double* lattices);

    // Evaluate from host buffers (positions already wrapped).  Blocking.
    void evaluate_host(const Damp& d, const double* positions, double* energies, double* gradient,
                       double* sigma9);
    // Evaluate from device buffers on `stream` (the caller's stream, used as
    // given: 0 is the legacy default stream).  Asynchronous.
    void evaluate_device(const Damp& d, const double* d_positions, double* d_energies,
                         double* d_gradient, double* d_sigma9, double* d_param_grad,
                         cudaStream_t stream);
    // Pairwise decomposition from host buffers (positions already wrapped),
    // FP64 and without the work partition (get_pairwise_dispersion_v2):
    // energy2 and energy3 receive [n_s][n_s] per system, one system after the
    // other.  Blocking.
    void pairwise_host(const Damp& d, const double* positions, double* energy2, double* energy3);
    // Analytic Hessian [3n][3n] of a batch of one structure from host
    // positions (already wrapped), FP64 (get_dispersion_hessian); the work
    // partition splits the pair and triple loops.  Blocking.
    void hessian_host(const Damp& d, const double* positions, double* hessian);

    cudaStream_t stream() const { return stream_; }

    // Captured launch sequence.  With the graph on, an evaluation replays one
    // CUDA graph of the whole pipeline (sort, CN, weights, two-body, three-body
    // lists and sum, chain rule, reductions) from engine-owned input/output
    // buffers.  The first evaluation of a (parameters, derivatives, tuning)
    // key runs the ordinary sequence, which sizes the three-body lists, and
    // then captures the graph with 25% headroom on those buffers; a replay
    // whose lists outgrow them is detected by a device flag and evaluated
    // again without the graph, and the graph is captured anew.
    void set_graph(bool on);
    bool graph() const { return graph_on_; }
    // kernel launches of one replay of the captured graph (0 before the first capture)
    long long graph_kernels() const { return graph_valid_ ? graph_kernels_ : 0; }

    // Partitioned evaluation over several processes (the reference's MPI
    // path, disp.f90:120-171 with a reducer, and mpi.f90): this engine
    // evaluates part `part` of `nparts` of every pair and triple loop,
    // including the CN and chain-rule loops, and calls `fn` to sum a device
    // buffer over all parts in place: the CN, then dE/dCN, then the results
    // [energies | parameter derivatives | virials | gradient] in one call.
    // `fn` is called on the host between launches and must order its work on
    // the given stream (a collective enqueued there, or a synchronisation
    // before a host exchange); it returns 0 on success.  All parts must have
    // the same systems, positions, parameters and launch shapes.  fn = null
    // ends the partition.  Not combinable with the captured graph.
    using Reducer = int (*)(double* buffer, int count, void* stream, void* user);
    void set_reducer(Reducer fn, void* user, int part, int nparts);

    // Launch shapes (spatial sort cell, atoms per pair block, resident triple
    // blocks per SM).  autotune() times the candidates on the given device
    // positions and keeps the fastest; it returns that time in ms.
    void set_tuning(const Tuning& t);
    const Tuning& tuning() const { return tune_; }
    double autotune(const Damp& d, const double* d_positions, bool grad, cudaStream_t stream);
    // Device buffer of natoms x 3 positions owned by the engine (autotune input).
    double* input_buffer();

    // Per-stage device times of the last evaluation (ms), recorded with CUDA
    // events when profiling is on.  Stages: see kStageNames.
    static constexpr int kStages = 7;
    // stage_times() also returns, after the stages, the time of the two-body
    // tile-pair kernel alone and of the three-body triple kernels alone
    static constexpr int kTimes = kStages + 2;
    void set_profiling(bool on) { profiling_ = on; }
    void stage_times(double out[kTimes]);

private:
    void build_tables(const int* numbers);
    void ensure_images(cudaStream_t stream);
    void ensure_workspace(bool grad, bool param_grad, bool threebody);
    void upload_pair_table(const Damp& d, cudaStream_t stream);
    void make_views(Batch& b, Species& s) const;
    bool cn_single_chunk() const;
    static constexpr size_t kCnStoreCap = size_t(768) << 20;   // bytes of stored chain-rule sums at most
    static constexpr int kFusedWeightsMaxAtoms = 65536;          // CN gather fused with weights and species vectors
    void* d_cn_store_ = nullptr;
    unsigned char* d_cn_store_ok_ = nullptr;
    size_t cn_store_cap_ = 0;
    void order_atoms(const Damp& d, const double* d_positions, const Batch& b, bool mixed, cudaStream_t stream);
    double* d_hs_ = nullptr;             // Hessian scratch and result
    double* d_rvdw_ = nullptr;           // [nid][nid] van der Waals radii (Hessian damping kernels)
    std::vector<int> img_off_host_;      // host copy of the image offsets
    double* d_pw_ = nullptr;             // pairwise decomposition: C6, energy2, energy3 (3 x sum n_s^2)
    long long* d_pw_off_ = nullptr;
    void run(const Damp& d, const double* d_positions, double* d_energies, double* d_gradient,
             double* d_sigma9, double* d_param_grad, bool grad, cudaStream_t stream);
    template <class T> T* dev_alloc(size_t n);

    void reduce(double* buffer, int count, cudaStream_t stream);
    Reducer reducer_ = nullptr;
    void* reducer_user_ = nullptr;
    double* d_red_ = nullptr;    // [nsys | 5 nsys | 9 nsys | 3 natoms] results of this part

    // graph state
    struct GraphKey {
        Damp damp;
        Cutoffs cut;
        Partition part;
        Tuning tune;
        int grad, pg, counting, mixed, cn_part;
    };
    GraphKey make_key(const Damp& d, bool grad, bool pg) const;
    void run_graphed(const Damp& d, bool grad, bool pg, cudaStream_t stream);
    void capture(const Damp& d, const GraphKey& key, bool grad, bool pg);
    void drop_graph();
    int atm_blocks(bool mixed, bool grad);      // resident triple blocks per SM (tuned)
    int atm_occupancy(bool mixed, bool grad);   // occupancy limit
    int atm_mol_occupancy(bool mixed, bool grad);
    int atm_mol_occ_[2][2] = {{0, 0}, {0, 0}};
    // two-body tile-pair units
    PairUnits pu_;
    int2* d_units_ = nullptr;
    int* d_unit_base_ = nullptr;
    std::vector<int> mol_order_;         // systems of the molecule kernel, largest first
    int* d_mol_order_ = nullptr;
    std::vector<int> sys_natoms_;
    int auto_split_ = 1;                 // pair split of tuning 0
    int pair_split() const;              // items per tile pair of the two-body sweep
    int cn_split() const;                // items per tile pair of the CN sweeps
    bool any_periodic_ = false;          // a system has a periodic direction
    void configure_molecules();          // mol_order_ and root_atoms_ from tune_.atm_mol
    // systems small enough for the direct pair kernels (see direct_pairs)
    static constexpr int kDirectMaxAtoms = DIRECT_MAX_ATOMS;
    static constexpr int kDirectMaxTotal = DIRECT_MAX_TOTAL;
    bool direct_pairs(const Damp& d, bool pg) const;
    uint8_t* d_sys_mol_ = nullptr;       // [nsys] 1 for those systems
    long long root_atoms_ = 0;           // atoms of the other systems
    bool graph_on_ = false, capturing_ = false, graph_valid_ = false;
    cudaGraphExec_t graph_exec_ = nullptr;
    long long graph_kernels_ = 0;
    GraphKey graph_key_{};
    unsigned long long alloc_epoch_ = 0, graph_epoch_ = 0;
    int* d_guard_ = nullptr;
    int* h_guard_ = nullptr;     // pinned
    int atm_stride_ = 0;         // reserved per-root list length of captured three-body sums
    double* d_pg_out_ = nullptr;
    Tuning tune_;
    int sms_ = 0;
    int atm_occ_[2][2] = {{0, 0}, {0, 0}};

    int device_ = 0;
    int nsys_ = 0, natoms_ = 0, max_sys_atoms_ = 0;
    std::vector<int> atom_off_, sys_of_atom_, local_, sp_;
    std::vector<int> zid_;               // species index inside the own system, from 1
    std::vector<double> lat_;
    std::vector<bool> per_storage_;
    std::unique_ptr<bool[]> per_;
    std::vector<uint8_t> ghost_;
    ModelTables tab_;
    Cutoffs cut_;
    Partition part_;
    bool cn_partitioned_ = false;
    bool mixed_ = false;
    bool counting_ = false;
    bool profiling_ = false;
    cudaEvent_t ev_[kStages + 1] = {};
    cudaEvent_t kev_[4] = {};            // two-body kernel, triple kernels: begin, end
    bool kev3_recorded_ = false;
    bool ev_recorded_ = false;
    bool images_valid_ = false;
    Damp last_damp_{};
    bool pair_valid_ = false;

    cudaStream_t stream_ = nullptr;
    std::vector<void*> allocations_;
    // static device data
    int *d_sys_of_atom_ = nullptr, *d_atom_off_ = nullptr, *d_local_ = nullptr, *d_sp_ = nullptr;
    uint8_t* d_ghost_ = nullptr;
    int* d_img_off_ = nullptr;
    double* d_img_ = nullptr;
    size_t img_capacity_ = 0;
    double *d_rcov_ = nullptr, *d_refcn_ = nullptr, *d_c6ref_ = nullptr, *d_pair_ = nullptr,
           *d_atm_r0_ = nullptr;
    float* d_c6ref_f_ = nullptr;
    int* d_nref_ = nullptr;
    // spatial order and tiles
    int ntiles_ = 0;
    int* d_tile_sys_ = nullptr;
    int* d_tile_off_ = nullptr;
    unsigned long long *d_keys_in_ = nullptr, *d_keys_out_ = nullptr;
    int *d_idx_in_ = nullptr, *d_perm_ = nullptr;
    int* d_identity_ = nullptr;           // 0 .. natoms - 1 (the order of the direct path)
    int *d_sp_sorted_ = nullptr, *d_local_sorted_ = nullptr, *d_zid_ = nullptr, *d_zid_sorted_ = nullptr;
    uint8_t* d_ghost_sorted_ = nullptr;
    double4* d_tiles_ = nullptr;
    int2* d_shape_ = nullptr;            // column order: slabs and columns per system
    void* d_sort_temp_ = nullptr;
    size_t sort_bytes_ = 0;
    // workspace
    double *d_x_ = nullptr, *d_y_ = nullptr, *d_z_ = nullptr;
    float4 *d_xhi_ = nullptr, *d_xlo_ = nullptr;
    Work work_{};
    bool ws_grad_ = false, ws_pg_ = false, ws_3b_ = false, ws_ready_ = false;
    double* d_pos_in_ = nullptr;
    double *d_energies_ = nullptr, *d_grad_out_ = nullptr, *d_sigma_ = nullptr;
    double *h_stage_ = nullptr;   // pinned staging: positions in, results out
    size_t h_stage_len_ = 0;
    unsigned long long* d_counts_ = nullptr;
    // three-body
    void run_three_body(const Batch& b, const Species& s, const Damp& d, const Config& c, Work& w,
                        cudaStream_t stream);
    void free_block(void*& p);
    std::vector<long long> c6mat_off_;
    long long c6mat_total_ = 0;
    long long* d_c6mat_off_ = nullptr;
    void* d_c6mat_ = nullptr;
    int* d_cnt_ = nullptr;
    long long* d_off_ = nullptr;
    int* d_maxcnt_ = nullptr;
    unsigned int* d_queue_ = nullptr;
    void* d_scan_temp_ = nullptr;
    size_t scan_bytes_ = 0;
    int* d_nbr_j_ = nullptr;
    int* d_nbr_gend_ = nullptr;
    double4* d_nbr_v_ = nullptr;
    long long nbr_cap_ = 0;
    double* d_slot_acc_ = nullptr;
    long long slot_cap_ = 0;
    void* d_slot_scr_ = nullptr;
    long long slot_scr_cap_ = 0;
    double* d_e3_ = nullptr;
    double* d_sig3_ = nullptr;
    unsigned long long* d_fxacc_ = nullptr;   // [natoms][4][2] fixed-point three-body gradient, dE/dCN
    long long* h_atm_counts_ = nullptr;   // pinned: total entries, largest list
    bool atm_ready_ = false;
    bool species_ready_ = false;   // PairUnits::U holds this evaluation's species vectors
    long long last_triples_entries_ = 0;
};

}  // namespace d3
