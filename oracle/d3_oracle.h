/* FP64 CPU oracle for the D3 dispersion hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * A loop-for-loop C restatement of the reference's Fortran algorithm, used by
 * the tests (as the parity checker), by __graft_entry__.smoke() and by
 * bench.py's CPU-baseline leg.  The product library never links or calls it.
 *
 * Parity is pinned against the reference's own golden vectors (see
 * tests/golden): validation fixtures, the Python API energies, the periodic Ta
 * regression and the AmF3 Gaussian-weight test. */
#pragma once

#ifdef __cplusplus
extern "C" {
#endif

/* damping families: rational (also the modified rational records), zero,
 * modified zero, optimized power, CSO and Z (src/dftd3/damping/) */
enum { ORACLE_RATIONAL = 0, ORACLE_ZERO = 1, ORACLE_MZERO = 2, ORACLE_OPTIMIZEDPOWER = 3,
       ORACLE_CSO = 4, ORACLE_Z = 5 };

typedef struct {
    int damping;      /* ORACLE_* */
    double s6, s8, s9;
    double a1, a2;    /* rational, optimized power, CSO, Z (a1) */
    double rs6, rs8;  /* zero, modified zero; CSO keeps a3 and a4 here as
                         new_cso_damping does (cso.f90:74-90) */
    double alp;
    double bet;       /* modified zero, optimized power */
} oracle_param;

typedef struct {
    double disp2, disp3, cn, width2, width3;
} oracle_cutoff;

/* Full evaluation, mirrors get_dispersion_atomic_v2 (disp.f90:56-185) with
 * the scalar energy of get_dispersion_scalar_v2 (disp.f90:352-399).
 *   numbers[nat], xyz[nat][3] (Bohr, already wrapped), lattice[3][3] with
 *   rows = lattice vectors, periodic[3] (0/1), ghost[nat] (0/1 or NULL).
 *   part/nparts: work partition (nparts <= 1: complete work); reduce_cn != 0
 *   partitions the coordination number like the reducer branch would.
 *   gradient[nat][3], sigma[3][3], energies[nat], cn[nat], dEdcn[nat] may be
 *   NULL.  Derivatives are computed when gradient or sigma is non-NULL.
 * Returns 0 on success, nonzero for unsupported elements or damping kinds. */
int oracle_get_dispersion(int nat, const int *numbers, const double *xyz,
                          const double *lattice, const int *periodic,
                          const int *ghost, const oracle_param *param,
                          const oracle_cutoff *cutoff, int part, int nparts,
                          double *energy, double *energies, double *gradient,
                          double *sigma, double *cn_out, double *dEdcn_out);

/* Pairwise decomposition, mirrors get_pairwise_dispersion_v2 (disp.f90:403-457):
 * pair2[nat][nat] the additive (two-body) and pair3[nat][nat] the
 * non-additive (three-body) energy of every atom pair; both sum to the
 * respective energy.  Returns 0 on success. */
int oracle_get_pairwise_dispersion(int nat, const int *numbers, const double *xyz,
                                   const double *lattice, const int *periodic, const int *ghost,
                                   const oracle_param *param, const oracle_cutoff *cutoff,
                                   double *pair2, double *pair3);

/* Analytic Hessian, mirrors get_dispersion_hessian (disp.f90:236-308):
 * hessian[3*nat][3*nat] (symmetric); part/nparts partition the pair and triple
 * loops as the reference does.  Returns 0 on success. */
int oracle_get_dispersion_hessian(int nat, const int *numbers, const double *xyz,
                                  const double *lattice, const int *periodic, const int *ghost,
                                  const oracle_param *param, const oracle_cutoff *cutoff,
                                  int part, int nparts, double *hessian);

/* In-place sum of count doubles over all parts; returns 0 on success. */
typedef int (*oracle_reducer)(double *buffer, int count, void *user);

/* The partitioned evaluation with a reducer (the reference's MPI path,
 * disp.f90:120-171 with `reducer`, and get_dispersion_mpi_atomic, mpi.f90):
 * part `part` of `nparts` evaluates its share of every pair and triple loop,
 * the CN and dE/dCN are summed over the parts before they are used, and the
 * atom energies, gradient and virial are summed at the end, so that every
 * part returns the complete result.  Returns 2 if the reducer failed. */
int oracle_get_dispersion_reduced(int nat, const int *numbers, const double *xyz,
                                  const double *lattice, const int *periodic, const int *ghost,
                                  const oracle_param *param, const oracle_cutoff *cutoff,
                                  int part, int nparts, oracle_reducer reduce, void *user,
                                  double *energy, double *energies, double *gradient, double *sigma);

/* Coordination numbers alone (ncoord.f90:86-144). */
int oracle_coordination_number(int nat, const int *numbers, const double *xyz,
                               const double *lattice, const int *periodic,
                               double cutoff, double *cn);

/* Gaussian reference weights for given CNs (model.f90:201-324), gwvec and
 * gwdcn laid out [nat][mref] with mref = max references over the species. */
int oracle_weight_references(int nat, const int *numbers, const double *cn,
                             int *mref_out, double *gwvec, double *gwdcn);

/* Lattice translations for a cutoff (cutoff.f90:140-227); returns the count
 * and, if trans is non-NULL and large enough (cap entries), fills trans[][3]. */
int oracle_lattice_points(const double *lattice, const int *periodic,
                          double rthr, double *trans, int cap);

/* Wrap positions into the central cell in place (utils.f90:29-64). */
void oracle_wrap_to_central_cell(int nat, double *xyz, const double *lattice,
                                 const int *periodic);

/* Per-element model data for checks of the tables. */
double oracle_covalent_radius(int z);
double oracle_r4r2(int z);

#ifdef __cplusplus
}
#endif
