/* Extensions of the B200 DFT-D3 library beyond the reference C API.
 *
 * None of these has a counterpart in the reference (s-dftd3 v1.6.0); they add
 * precision selection, ragged batches of independent systems in one
 * evaluation, and an entry point on device buffers for framework callers
 * (the torch autograd wrapper).  Handles and the error convention are those of
 * s-dftd3.h. */
#pragma once

#include "s-dftd3.h"

/* Arithmetic of the hot path: FP64 everywhere (the default, parity form), or
 * FP32 pair/triple arithmetic with FP64 accumulation, weights and reductions. */
#define DFTD3_B200_PRECISION_FP64 0
#define DFTD3_B200_PRECISION_MIXED 1

typedef struct _dftd3_b200_batch* dftd3_b200_batch;

/* Launch shapes of a model created by dftd3_new_d3_model (tuning[4] as for
 * dftd3_b200_set_batch_tuning). */
SDFTD3_API_ENTRY void SDFTD3_API_CALL
dftd3_b200_set_model_tuning(dftd3_error /* error */,
                            dftd3_model /* model */,
                            const double* /* tuning[4] */);

/* Select the arithmetic of a model created by dftd3_new_d3_model. */
SDFTD3_API_ENTRY void SDFTD3_API_CALL
dftd3_b200_set_model_precision(dftd3_error /* error */,
                               dftd3_model /* model */,
                               int /* precision */);

/* Replay the evaluation of a model created by dftd3_new_d3_model as one
 * captured CUDA graph (enable != 0), as dftd3_b200_set_batch_graph does for a
 * batch: the first dftd3_get_dispersion after enabling captures, later calls
 * with new positions replay it. */
SDFTD3_API_ENTRY void SDFTD3_API_CALL
dftd3_b200_set_model_graph(dftd3_error /* error */,
                           dftd3_model /* model */,
                           int /* enable */);

/* Create a batch of nsys independent systems.  Atoms are concatenated:
 * natoms[nsys], numbers[sum natoms].  lattices[nsys][3][3] and
 * periodic[nsys][3] may be NULL for molecules.  The batch keeps device
 * workspace and the captured launch sequence between evaluations. */
SDFTD3_API_ENTRY dftd3_b200_batch SDFTD3_API_CALL
dftd3_b200_new_batch(dftd3_error /* error */,
                     int /* nsys */,
                     const int* /* natoms [nsys] */,
                     const int* /* numbers [sum natoms] */,
                     const double* /* lattices [nsys][3][3] or NULL */,
                     const bool* /* periodic [nsys][3] or NULL */);

SDFTD3_API_ENTRY void SDFTD3_API_CALL
dftd3_b200_set_batch_realspace_cutoff(dftd3_error /* error */,
                                      dftd3_b200_batch /* batch */,
                                      double /* disp2 */,
                                      double /* disp3 */,
                                      double /* cn */,
                                      double /* width2 */,
                                      double /* width3 */);

SDFTD3_API_ENTRY void SDFTD3_API_CALL
dftd3_b200_set_batch_precision(dftd3_error /* error */,
                               dftd3_b200_batch /* batch */,
                               int /* precision */);

/* Evaluate all systems from host buffers.  positions[sum natoms][3] (Bohr) are
 * wrapped per system like dftd3_new_structure; lattices may be NULL to keep
 * the batch's lattices.  energies[nsys]; gradient[sum natoms][3] and
 * sigma[nsys][3][3] may be NULL (then only energies are evaluated). */
SDFTD3_API_ENTRY void SDFTD3_API_CALL
dftd3_b200_get_dispersion_batched(dftd3_error /* error */,
                                  dftd3_b200_batch /* batch */,
                                  dftd3_param /* param */,
                                  const double* /* positions */,
                                  const double* /* lattices or NULL */,
                                  double* /* energies [nsys] */,
                                  double* /* gradient [sum natoms][3] or NULL */,
                                  double* /* sigma [nsys][3][3] or NULL */);

/* Evaluate all systems from device buffers on the caller's stream (a
 * cudaStream_t used as given; NULL is the legacy default stream).  Positions are used as
 * given (no wrapping); the lattices, which decide the image lists, are read
 * from host memory (NULL keeps the current ones).  param_grad[nsys][5], if
 * non-NULL, receives
 * dE/d(s6, s8, a1, a2, s9) (rational) or dE/d(s6, s8, rs6, rs8, s9) (zero).
 * Two-body evaluations are asynchronous with respect to the host.  With the
 * three-body term the call waits for the device once: for the neighbour
 * list sizes (ordinary sequence) or for the list capacity check at the end
 * (captured sequence, dftd3_b200_set_batch_graph). */
SDFTD3_API_ENTRY void SDFTD3_API_CALL
dftd3_b200_get_dispersion_device(dftd3_error /* error */,
                                 dftd3_b200_batch /* batch */,
                                 dftd3_param /* param */,
                                 const double* /* d_positions [sum natoms][3] */,
                                 const double* /* lattices [nsys][3][3] (host) or NULL */,
                                 double* /* d_energies [nsys] */,
                                 double* /* d_gradient or NULL */,
                                 double* /* d_sigma or NULL */,
                                 double* /* d_param_grad or NULL */,
                                 void* /* stream */);

/* Work counters of the last evaluation: accepted pair terms of the two-body
 * sum, accepted ATM triples and CN terms (counted on request, see
 * dftd3_b200_set_batch_counting). */
SDFTD3_API_ENTRY void SDFTD3_API_CALL
dftd3_b200_set_batch_counting(dftd3_error /* error */,
                              dftd3_b200_batch /* batch */,
                              int /* enable */);

SDFTD3_API_ENTRY void SDFTD3_API_CALL
dftd3_b200_get_batch_counts(dftd3_error /* error */,
                            dftd3_b200_batch /* batch */,
                            long long* /* counts[3]: pair, triple, cn */);

/* Device time of each pipeline stage of the last evaluation in ms, recorded
 * with CUDA events while profiling is enabled: [0] position split, [1]
 * coordination number, [2] reference weights, [3] two-body, [4] three-body,
 * [5] CN chain rule, [6] per-system reductions; then [7] the two-body
 * tile-pair kernel alone and [8] the three-body triple kernels alone (0 when
 * not run). */
SDFTD3_API_ENTRY void SDFTD3_API_CALL
dftd3_b200_set_batch_profiling(dftd3_error /* error */,
                               dftd3_b200_batch /* batch */,
                               int /* enable */);

SDFTD3_API_ENTRY void SDFTD3_API_CALL
dftd3_b200_get_batch_stage_times(dftd3_error /* error */,
                                 dftd3_b200_batch /* batch */,
                                 double* /* ms[9] */);

/* Kernel launches of one replay of the batch's captured CUDA graph: the
 * kernel nodes of the graph (0 while no graph is captured). */
SDFTD3_API_ENTRY void SDFTD3_API_CALL
dftd3_b200_get_batch_graph_kernels(dftd3_error /* error */,
                                   dftd3_b200_batch /* batch */,
                                   long long* /* kernels */);

/* Replay the whole pipeline of an evaluation as one captured CUDA graph
 * (enable != 0).  The first evaluation for a parameter set, derivative set
 * and launch shape runs the ordinary launch sequence and then captures it;
 * later evaluations launch the graph on the caller's stream.  Inputs and
 * outputs are staged through buffers the batch owns.  Per-stage times are
 * not recorded for graph replays.  A replay whose three-body lists outgrow
 * the captured buffers is detected and evaluated again without the graph. */
SDFTD3_API_ENTRY void SDFTD3_API_CALL
dftd3_b200_set_batch_graph(dftd3_error /* error */,
                           dftd3_b200_batch /* batch */,
                           int /* enable */);

/* Launch shapes of a batch: tuning[0] the spatial order of the atoms (0:
 * column order, tiles of 32 atoms cut from slabs and columns of each system,
 * the default, Morton order with 3 Bohr cells for systems above 16384 atoms;
 * > 0: Morton order with keys quantised to cells of that many Bohr),
 * tuning[1] work items per tile pair of the pair sweeps (1, 2
 * or 4; 0 chooses 1 for batches of molecules, else 2, and 1 for the CN
 * sweeps of the mixed form when the tile pairs give every SM eight warps),
 * tuning[2] resident blocks per SM of the neighbour-list three-body
 * kernel (0 = occupancy limit), tuning[3] the block-per-molecule three-body
 * kernel for non-periodic systems of at most 256 atoms (0: when the batch has
 * at least one such molecule per SM, 1: always, 2: never). */
SDFTD3_API_ENTRY void SDFTD3_API_CALL
dftd3_b200_set_batch_tuning(dftd3_error /* error */,
                            dftd3_b200_batch /* batch */,
                            const double* /* tuning[4] */);

SDFTD3_API_ENTRY void SDFTD3_API_CALL
dftd3_b200_get_batch_tuning(dftd3_error /* error */,
                            dftd3_b200_batch /* batch */,
                            double* /* tuning[4] */);

/* Autotuner: time the candidate launch shapes on these positions (host,
 * [sum natoms][3], wrapped like dftd3_b200_get_dispersion_batched) with the
 * gradient on or off, keep the fastest shape and return its time in ms. */
SDFTD3_API_ENTRY double SDFTD3_API_CALL
dftd3_b200_autotune_batch(dftd3_error /* error */,
                          dftd3_b200_batch /* batch */,
                          dftd3_param /* param */,
                          const double* /* positions */,
                          int /* gradient */);

/* Reducer of a partitioned evaluation: sums `count` doubles of a device
 * buffer in place over all parts (an all-reduce over the processes of a
 * job).  Called on the host between kernel launches with the stream of the
 * evaluation; it must order its work on that stream (for example a NCCL
 * all-reduce enqueued there, or a stream synchronisation before a host
 * exchange) and return 0 on success. */
typedef int (*dftd3_b200_reducer)(double* /* buffer */,
                                  int /* count */,
                                  void* /* stream */,
                                  void* /* user data */);

/* Distribute the evaluation of a batch over nparts processes, this one
 * being part `part` (0-based): the stand-in for dftd3_set_model_mpi_comm
 * (reference api.f90:483-506) for callers that own their communicator (NCCL
 * through torch.distributed, MPI, ...).  Every pair and triple loop,
 * including the coordination number and its chain rule, is split by the
 * reference's pair ownership (partition.f90:127-147); the coordination
 * numbers and dE/dCN are summed over the parts before they are used
 * (disp.f90:120-126,166-171) and the results once at the end
 * (get_dispersion_mpi_atomic, mpi.f90), so every part returns the complete
 * energies, gradient and virials.  All parts must evaluate the same
 * positions, parameters and launch shapes.  reducer = NULL ends the
 * partition.  Not combinable with dftd3_b200_set_batch_graph. */
SDFTD3_API_ENTRY void SDFTD3_API_CALL
dftd3_b200_set_batch_reducer(dftd3_error /* error */,
                             dftd3_b200_batch /* batch */,
                             dftd3_b200_reducer /* reducer or NULL */,
                             void* /* user data */,
                             int /* part */,
                             int /* nparts */);

SDFTD3_API_ENTRY void SDFTD3_API_CALL
dftd3_b200_delete_batch(dftd3_b200_batch* /* batch */);

/* Energy, gradient and virial of one system (two-body term, s9 = 0) without
 * allocating memory.  This entry point has no counterpart in the reference.
 * It serves callers that cannot allocate device memory while they run --
 * integrators and MD engines that hand out all device memory from their own
 * pool, time-step loops in which cudaMalloc/cudaFree (which can synchronise
 * the device) are not allowed.  All work arrays come from a fixed __device__
 * array inside the library (4 MiB), held by every GPU that loads it until
 * exit.  The call copies small per-call tables from static host buffers on
 * `stream` and waits for that stream before returning (so it blocks the host
 * until earlier work on `stream` is done); the kernels then run
 * asynchronously.  A CUDA launch error pending from earlier work is reported
 * and nothing is launched; periodic directions need a non-degenerate lattice.
 *   numbers[natoms], lattice[3][3], periodic[3] and cutoffs[5] (disp2, disp3,
 *   cn, width2, width3; NULL for the defaults) are host memory;
 *   d_positions[natoms][3], d_energy[1], d_gradient[natoms][3] and
 *   d_sigma[9] are device memory (gradient and sigma may be NULL); positions
 *   are used as given (no wrapping).  Work is enqueued on `stream`.
 * Limits: 4096 atoms, 16 elements, 8192 lattice translations per cutoff;
 * larger inputs are rejected with an error.  All calls on a device share the
 * array, so calls that overlap on the GPU race and must be serialised by the
 * caller.  The first call on a device looks up the array's device address
 * with that device current; make it before any stream capture. */
SDFTD3_API_ENTRY void SDFTD3_API_CALL
dftd3_b200_get_dispersion_noalloc(dftd3_error /* error */,
                                  dftd3_param /* param */,
                                  int /* natoms */,
                                  const int* /* numbers [natoms] (host) */,
                                  const double* /* d_positions [natoms][3] */,
                                  const double* /* lattice [3][3] (host) or NULL */,
                                  const bool* /* periodic [3] (host) or NULL */,
                                  const double* /* cutoffs [5] (host) or NULL */,
                                  int /* precision */,
                                  double* /* d_energy [1] */,
                                  double* /* d_gradient [natoms][3] or NULL */,
                                  double* /* d_sigma [9] or NULL */,
                                  void* /* stream */);

/* Damping families of a parameter handle (dftd3_b200_get_param_values);
 * the modified rational records are evaluated with the rational form. */
#define DFTD3_B200_DAMPING_RATIONAL 0
#define DFTD3_B200_DAMPING_ZERO 1
#define DFTD3_B200_DAMPING_MZERO 2
#define DFTD3_B200_DAMPING_OPTIMIZEDPOWER 3
#define DFTD3_B200_DAMPING_CSO 4
#define DFTD3_B200_DAMPING_Z 5

/* Values of a damping parameter handle: *kind one of DFTD3_B200_DAMPING_*;
 * values[9] = s6, s8, s9, a1, a2, rs6, rs8, alp, bet (CSO: a3 and a4 in the
 * rs6 and rs8 places, as the reference's d3_param record holds them).  For
 * inspecting parameters loaded by method name (dftd3_load_*_damping). */
SDFTD3_API_ENTRY void SDFTD3_API_CALL
dftd3_b200_get_param_values(dftd3_error /* error */,
                            dftd3_param /* param */,
                            int* /* kind */,
                            double* /* values[9] */);

/* Measured fused-multiply-add throughput of the current device in TFLOP/s
 * (precision DFTD3_B200_PRECISION_FP64: FP64 pipe, _MIXED: FP32 pipe); the
 * denominator of the roofline fraction the benchmark reports. */
SDFTD3_API_ENTRY double SDFTD3_API_CALL
dftd3_b200_fma_peak(dftd3_error /* error */,
                    int /* precision */);
