// Device-side data layout of the D3 pipeline and the kernel entry points.
//
// One evaluation covers a ragged batch of independent systems.  Atoms of all
// systems are concatenated; every per-atom array below is indexed by the
// batch atom index.  A single structure is a batch of one.
#pragma once

#include <cuda_runtime.h>
#include <cfloat>
#include <cmath>
#include <cstdint>

namespace d3 {

// Programmatic dependent launch: the pipeline kernels are launched with
// launch_pdl, so that the launch of the next kernel overlaps the end of the
// current one, and every such kernel starts with pdl_wait() (the predecessor
// grid has completed and its memory is visible) before it touches global
// memory.  The kernels do not signal their successors early: under graph
// replay an early signal let the next kernel's blocks take SM slots from the
// current kernel's last wave (0.293 -> 0.300 ms on the headline step), while
// the plain form still takes the ordinary-launch evaluation of a 100-atom
// molecule from 84 to 76 us.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

template <typename... KArgs, typename... Args>
inline void launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t stream,
                       Args... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

constexpr int kMaxRef = 7;          // references per element (reference.f90:28)
constexpr int kImageKinds = 3;      // lattice point sets: CN, two-body, three-body
constexpr int kImgCN = 0, kImgDisp2 = 1, kImgDisp3 = 2;
constexpr int kSigma = 6;           // packed symmetric virial: xx yy zz xy xz yz
constexpr int kParamGrad = 5;       // dE/d(s6, s8, a1|rs6, a2|rs8, s9)
constexpr int kPairSlots = 6;       // per species pair: rrij, q1..q5 (family constants)
constexpr int kRefPad = 8;          // species-vector stride: U[0..6], pad, dU[0..6], pad

// Damping families of the two-body sum (src/dftd3/damping/); the modified
// rational records are evaluated with kRational.
enum Damping : int { kRational = 0, kZero = 1, kMZero = 2, kOptimizedPower = 3, kCSO = 4, kZDamping = 5 };
constexpr int kDampingKinds = 6;
// families with dE/d(damping parameter) in the kernels
inline bool damping_has_param_grad(int kind) { return kind == kRational || kind == kZero; }

// Per-batch geometry and bookkeeping.
struct Batch {
    int nsys = 0, natoms = 0, nid = 0;
    const int* sys_of_atom = nullptr;    // [natoms]
    const int* atom_off = nullptr;       // [nsys + 1]
    const int* local = nullptr;          // [natoms] index inside its system
    const int* sp = nullptr;             // [natoms] batch species index
    const int* zid = nullptr;            // [natoms] species index inside its own system, from 1
                                         // (first occurrence; the Z damping's mol%id)
    const uint8_t* ghost = nullptr;      // [natoms] or null
    const int* img_off = nullptr;        // [kImageKinds][nsys + 1]
    const double* img = nullptr;         // [nimg][3]
    const double* x = nullptr;           // [natoms] SoA positions (Bohr)
    const double* y = nullptr;
    const double* z = nullptr;
    const float4* xhi = nullptr;         // [natoms] float head of x,y,z (mixed form)
    const float4* xlo = nullptr;         // [natoms] float tail x - head
    // spatial order (optional): atom slot a holds the input atom perm[a]; the
    // per-atom arrays above are then in slot order
    const int* perm = nullptr;           // [natoms] or null (input order)
    const double4* tiles = nullptr;      // [ntiles] bounding sphere (centre, radius) of 32 slots, or null
    const int* tile_off = nullptr;       // [nsys + 1] first tile of each system
    const int* tile_sys = nullptr;       // [ntiles] system of each tile
};

// Tile-pair work units of the two-body sum (d3_pair_tt.cu): for every
// system, the pairs (it >= jt) of its tiles in the order it = 0.., jt = 0..it,
// starting at unit_base[sys]; per-unit slots of kTile lanes.
struct PairUnits {
    const int2* units = nullptr;         // [nunits] global tile indices (it, jt)
    int nunits = 0;
    const int* unit_base = nullptr;      // [nsys]
    int split = 4;                       // items per unit: 1, 2 (j-tile halves), 4 (and translation halves)
    bool single_image = false;           // every system has the lattice point T = 0 only (molecules) and
                                         // the two-body sum takes the diagonal walk (k_two_body_rot)
    void* U = nullptr;                   // [natoms][nid][16] species vectors U (7 + pad) and dU (7 + pad) (R)
    double* unit_i = nullptr;            // [nunits][kTile][15]
    double* unit_j = nullptr;            // [nunits][kTile][4]
    // chain-rule sums of the CN pass per (item, j, lane), or null: the CN
    // pass stores them and the chain rule reads them instead of evaluating
    // the terms again (systems of one translation chunk, cn_store_bytes)
    void* cn_store = nullptr;            // [items][kTile / splitJ][3][kTile] (R)
    unsigned char* cn_store_ok = nullptr;   // [items]: the item stored its sums
};

constexpr int kTile = 32;               // atoms per tile (one warp)
constexpr int kMaxSpeciesFast = 16;     // species handled by the culled pair kernels

// Per-species model tables (new_d3_model, model.f90:87-181) for the batch's
// species set, and the per-pair damping constants of the current parameters.
struct Species {
    const double* rcov = nullptr;        // [nid]
    const int* nref = nullptr;           // [nid]
    const double* refcn = nullptr;       // [nid][kMaxRef]
    const double* c6ref = nullptr;       // [nid][nid][kMaxRef][kMaxRef] = c6(ir, jr, is, js)
    const float* c6ref_f = nullptr;      // same in FP32 (mixed form)
    const double* pair = nullptr;        // [nid][nid][kPairSlots] damping constants, see engine
    const double* atm_r0 = nullptr;      // [nid][nid] rs9 * rvdw
};

// Damping parameters (the reference's d3_param record, param.f90:38-48):
// CSO keeps its a3 and a4 in rs6 and rs8 as new_cso_damping does
// (cso.f90:74-90); bet belongs to the modified zero and optimized power forms.
struct Damp {
    int kind = kRational;
    double s6 = 1, s8 = 1, s9 = 0, a1 = 0.4, a2 = 5, rs6 = 1, rs8 = 1, alp = 14, bet = 0;
};

// Whether the two-body sum contributes: the early return of each family's
// get_dispersion2 (rational.f90:266, cso.f90:223 tests s6 and a1).
inline bool two_body_active(const Damp& d)
{
    if (d.kind == kCSO) return std::fabs(d.s6) >= DBL_EPSILON || std::fabs(d.a1) >= DBL_EPSILON;
    return std::fabs(d.s6) >= DBL_EPSILON || std::fabs(d.s8) >= DBL_EPSILON;
}

struct Partition {
    int part = 0, nparts = 1;
};

// Work arrays of one evaluation.
struct Work {
    double* cn = nullptr;        // [natoms]
    double* gw = nullptr;        // [natoms][kMaxRef]
    double* dgw = nullptr;       // [natoms][kMaxRef]
    float* gwf = nullptr;        // [natoms][kMaxRef] (mixed form)
    float* dgwf = nullptr;       // [natoms][kMaxRef] (mixed form)
    double* dEdcn = nullptr;     // [natoms]
    double* e_atom = nullptr;    // [natoms]
    double* grad = nullptr;      // [natoms][3]
    double* sig_atom = nullptr;  // [natoms][kSigma]
    double* cn_sig = nullptr;    // [natoms][kSigma] sum of the CN chain rule's countd v^T over the atom's
                                 // pairs (the stored-sum CN pass; virial = sum dE/dCN_i cn_sig_i)
    double* pg_atom = nullptr;   // [natoms][kParamGrad] or null
    unsigned long long* counts = nullptr;  // [3] pair, triple, cn terms or null
    // three-body results per root atom (summed by the per-system reduction)
    double* e3_atom = nullptr;   // [natoms] three-body energy of the root's triples
    double* sig3_atom = nullptr; // [natoms][kSigma] three-body virial of the root's triples
    // dE/ds9 of the parameter derivatives: pg_s9_scale * sum of e3_pg (the
    // three-body energy at the current s9, or at s9 = 1 when s9 vanishes)
    const double* e3_pg = nullptr;
    double pg_s9_scale = 0.0;
    // capacity guard of the three-body lists: set when the neighbour entries
    // exceed the reserved buffers (captured launch sequences); the list fill
    // and the triple sum then skip their work
    int* atm_guard = nullptr;
};

struct Config {
    double cut_cn = 40, cut2 = 60, cut3 = 40, width2 = 0, width3 = 0;
    bool grad = true;
    bool mixed = false;
    bool param_grad = false;
    bool cn_partitioned = false;   // partition the CN and chain-rule loops too
    int pair_warps = 8;            // atoms (warps) per block of the culled pair sweeps: 4 or 8
};

// Launch-shape choices of one batch, picked by the autotuner or set by hand.
struct Tuning {
    double morton_cell = 0.0;      // spatial order: 0 = column order (compact tiles; Morton with 3 Bohr
                                   // cells for systems above kRankOrderMax atoms), > 0 = Morton order
                                   // with keys quantised to cells of this many Bohr
    int pair_split = 0;            // work items per tile pair of the pair sweeps: 1, 2 or 4; 0 = 1 for
                                   // molecules, else 2 (mixed form) or 4 (FP64 form)
    int atm_blocks_per_sm = 0;     // resident blocks per SM of the neighbour-list triple kernel; 0 = occupancy
    int atm_mol = 0;               // molecule triple kernel: 0 for batches of at least one molecule per SM,
                                   // 1 for every eligible system, 2 never
};

// Pairwise decomposition (d3_pairwise.cu), FP64: energy2 and energy3 of every
// system as [n_s][n_s] blocks at off[sys] (input atom order); c6 is scratch of
// the same size.  Needs the sorted atoms and the reference weights.
void launch_pairwise(const Batch& b, const Species& s, const Damp& d, const Config& c, const Work& w,
                     const long long* off, long long total, double* c6, double* e2, double* e3,
                     cudaStream_t stream);

// Analytic Hessian of one structure (d3_hessian.cu), FP64, input atom order:
// pos [n][3], sp, zid, ghost per atom; img_range = the [first, last) image
// indices of the CN, two-body and three-body lattice points; rvdw [nid][nid];
// scratch of hessian_scratch_doubles(n); H [3n][3n].
size_t hessian_scratch_doubles(int n);
void launch_hessian(const Species& s, const Damp& d, const Config& c, const Partition& p, int n, int nid,
                    const double* pos, const int* sp, const int* zid, const uint8_t* ghost, const double* img,
                    const int img_range[6], const double* rvdw, double* scratch, double* H, cudaStream_t stream);

// FMA throughput of the FP64 (fp64=true) or FP32 pipe in TFLOP/s (blocking).
double measure_fma_peak(bool fp64);

// Launchers (d3_kernels.cu); all asynchronous on `stream`.
void launch_split_positions(const double* pos, int natoms, double* x, double* y, double* z,
                            float4* xhi, float4* xlo, bool mixed, cudaStream_t stream);
// Atoms in input order (small systems): the CN kernel reads the positions
// from the input array, writes the batch's position arrays (x, y, z and, in
// the mixed form, the FP32 head and tail) and goes on with the reference
// weights and, into uv (natoms x nid x 2 x kRefPad of the form's type), the
// species vectors.
struct InputPositions {
    const double* pos = nullptr;   // [natoms][3]
    double* x = nullptr;
    double* y = nullptr;
    double* z = nullptr;
    float4* xhi = nullptr;
    float4* xlo = nullptr;
};
void launch_coordination_number(const Batch& b, const Species& s, const Config& c,
                                const Partition& p, const Work& w, cudaStream_t stream,
                                const InputPositions* in = nullptr, void* uv = nullptr);
void launch_weights(const Batch& b, const Species& s, const Config& c, const Work& w,
                    cudaStream_t stream);
void launch_two_body(const Batch& b, const Species& s, const Damp& d, const Config& c,
                     const Partition& p, const Work& w, cudaStream_t stream,
                     const void* uv = nullptr);
// Spatial ordering and tile bounds (d3_pair.cu).
size_t sort_temp_bytes(int natoms);
void launch_spatial_sort(const double* pos, int natoms, const int* sys_of_atom, double cell,
                         unsigned long long* keys_in, unsigned long long* keys_out, int* idx_in, int* perm,
                         void* temp, size_t temp_bytes, cudaStream_t stream);
// Column order (the default; d3_pair.cu) of batches whose systems have at
// most kRankOrderMax atoms: per system nx slabs x ny columns of whole tiles,
// z inside a column, by ranks; writes perm and the sorted atom arrays (the
// tile bounds follow with launch_tile_bounds).  shape: [nsys], word_a and
// word_b: [natoms] scratch.
constexpr int kRankOrderMax = 16384;
void launch_rank_order(const double* pos, int natoms, int nsys, int max_atoms, const int* sys_of_atom,
                       const int* atom_off, const int* tile_off, int2* shape, unsigned long long* word_a,
                       unsigned long long* word_b,
                       const int* sp_in, const uint8_t* ghost_in, const int* zid_in, bool mixed, int* perm,
                       double* x, double* y, double* z, float4* xhi, float4* xlo, int* sp, uint8_t* ghost,
                       int* local, int* zid, cudaStream_t stream);
void launch_gather_sorted(const double* pos, const int* perm, const int* sp_in, const uint8_t* ghost_in,
                          const int* sys_of_atom, const int* atom_off, int natoms, double* x, double* y,
                          double* z, float4* xhi, float4* xlo, int* sp, uint8_t* ghost, int* local, bool mixed,
                          cudaStream_t stream, const int* zid_in = nullptr, int* zid = nullptr);
void launch_tile_bounds(const Batch& b, const int* tile_sys, int ntiles, double4* tiles, cudaStream_t stream);
// The same column order, sorted atom arrays and tile bounds by one block per
// system (three bitonic sorts in shared memory, one launch) for batches of at
// least kOrderBlockMinSystems systems of at most kOrderBlockMax atoms.
constexpr int kOrderBlockMax = 4096;
constexpr int kOrderBlockMinSystems = 32;
void launch_order_block(const double* pos, int nsys, int max_atoms, const int* atom_off, const int* tile_off,
                        const int* sp_in, const uint8_t* ghost_in, const int* zid_in, bool mixed, int* perm,
                        double* x, double* y, double* z, float4* xhi, float4* xlo, int* sp, uint8_t* ghost,
                        int* local, int* zid, double4* tiles, cudaStream_t stream);
// Culled pair sweeps over sorted atoms and tiles (d3_pair.cu); used by the
// launchers below when b.tiles is set and nid <= kMaxSpeciesFast.
void launch_coordination_number_tiled(const Batch& b, const Species& s, const Config& c, const Partition& p,
                                      const Work& w, cudaStream_t stream);
void launch_two_body_tiled(const Batch& b, const Species& s, const Damp& d, const Config& c, const Partition& p,
                           const Work& w, cudaStream_t stream);
void launch_cn_chain_rule_tiled(const Batch& b, const Species& s, const Config& c, const Partition& p,
                                const Work& w, cudaStream_t stream);

// Two-body sum over tile-pair units, each atom pair once, with the per-atom
// gather (d3_pair_tt.cu); writes e_atom, dEdcn, grad, sig_atom, pg_atom.
// Coordination number (chain = false, writes cn) or its chain rule (chain =
// true, adds to grad and sig_atom) over the same units (d3_pair_tt.cu).
// weights: the CN pass also writes the reference weights (as launch_weights)
// and, when uv is given, the species vectors of PairUnits::U.
size_t cn_store_bytes(const PairUnits& pu, bool mixed);   // d3_pair_tt.cu
constexpr int kCnStoreChunk = 128; // translations of a system the stored chain rule covers
void launch_cn_units(const Batch& b, const Species& s, const Config& c, const Partition& p, const Work& w,
                     const PairUnits& pu, bool chain, cudaStream_t stream, bool weights = false, void* uv = nullptr);
size_t pair_unit_slot_doubles();   // per unit: i and j slots
size_t pair_unit_i_doubles();      // per unit: i slots
size_t species_vector_doubles(int natoms, int nid);   // PairUnits::U (FP64 size)
// Species vectors U[a][s][r] = sum_q C6ref(r of s, q of atom a's species) gw_a[q]
// and dU with dgw (zero for ghosts), in the arithmetic type of the form.
void launch_species_vectors(const Batch& b, const Species& s, const Config& c, const Work& w, void* U,
                            cudaStream_t stream);
// ev_begin/ev_end (or null) are recorded around the tile-pair kernel alone;
// species_ready: the CN pass wrote the species vectors.
void launch_two_body_units(const Batch& b, const Species& s, const Damp& d, const Config& c, const Partition& p,
                           const Work& w, const PairUnits& pu, cudaStream_t stream, cudaEvent_t ev_begin = nullptr,
                           cudaEvent_t ev_end = nullptr, bool species_ready = false);

// Three-body term (d3_atm.cu): C6 table, neighbour lists, triple sum.
size_t atm_c6_entry_bytes(bool mixed);
// From the species vectors U (launch_species_vectors) and the weights.
void launch_c6_matrix(const Batch& b, const Species& s, const Work& w, const void* U, double alp3,
                      const long long* d_mat_off, void* mat, long long total, bool mixed, cudaStream_t stream);
// sys_skip[nsys] (or null): systems whose roots get no entries (handled by
// the molecule kernel)
void launch_nbr_count(const Batch& b, const Config& c, const uint8_t* sys_skip, int* cnt, int* max_cnt,
                      cudaStream_t stream);
size_t scan_temp_bytes(int n);
void launch_scan(void* temp, size_t temp_bytes, const int* cnt_ext, long long* off, int n,
                 cudaStream_t stream);
// Sets *guard when off[natoms] (the entry total) exceeds cap or the longest
// list exceeds stride; the fill and triple kernels then return at once.
void launch_atm_guard(const long long* total, const int* max_cnt, long long cap, int stride, int* guard,
                      cudaStream_t stream);
void launch_nbr_fill(const Batch& b, const Config& c, const uint8_t* sys_skip, const long long* off, const int* cnt,
                     int* nbr_j, int* nbr_gend, double4* nbr_v, const int* guard, cudaStream_t stream);
int atm_blocks_per_sm(bool mixed, bool grad);
size_t atm_slot_bytes(bool mixed);
// With gradients the force and dE/dCN share of every entry's atom and of the
// root go to fxacc[natoms][4][2] (fixed point, zeroed before the launch);
// launch_atm_fixed then adds them to the gradient and dE/dCN.
void launch_triples(const Batch& b, const Species& s, const Damp& d, const Config& c, const Partition& p,
                    const Work& w, const void* mat, const long long* mat_off, const long long* off,
                    const int* cnt, const int* nbr_j, const int* nbr_gend, const double4* nbr_v,
                    unsigned int* queue, double* slot_acc, void* slot_scr, int slot_stride, int blocks,
                    bool periodic, double* e3, double* sig3, unsigned long long* fxacc, cudaStream_t stream);
void launch_atm_fixed(int natoms, const unsigned long long* fxacc, const int* guard, const Work& w,
                      cudaStream_t stream);
// Three-body term of whole molecules, one block per system (d3_atm_mol.cu):
// the non-periodic systems of at most atm_mol_max_atoms() atoms listed in
// mol_order (largest first).  Writes e3/sig3 for every atom of those systems.
int atm_mol_max_atoms();
int atm_mol_blocks_per_sm(bool mixed, bool grad);
void launch_triples_mol(const Batch& b, const Species& s, const Damp& d, const Config& c, const Partition& p,
                        const Work& w, const void* mat, const long long* mat_off, const int* mol_order, int nmol,
                        unsigned int* queue, int blocks, double* e3, double* sig3, cudaStream_t stream);
void launch_cn_chain_rule(const Batch& b, const Species& s, const Config& c, const Partition& p,
                          const Work& w, cudaStream_t stream,
                          bool direct = false);
void launch_reduce_systems(const Batch& b, const Config& c, const Work& w, double* energies,
                           double* sigma9, double* param_grad, double* grad_out,
                           cudaStream_t stream);

}  // namespace d3
