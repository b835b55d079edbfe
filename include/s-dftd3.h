/* C API of the B200 DFT-D3 dispersion library.
 *
 * Drop-in for the reference's public header (include/s-dftd3.h of
 * s-dftd3 v1.6.0): every entry point below has the reference's name,
 * signature, argument meaning and error convention, and each comment names
 * the reference implementation it replaces (src/dftd3/api.f90).  Entry
 * points outside the dispersion hot path link and report "not supported"
 * through the error handle.
 *
 * Units are atomic units: Bohr in, Hartree and Hartree/Bohr out.  Arrays are
 * C-contiguous: positions[natoms][3], lattice[3][3] with one lattice vector per
 * row, gradient[natoms][3], sigma[3][3] in the reference's (Fortran) order.
 *
 * Additive extensions (batched and device-pointer evaluation, precision
 * selection) are declared in dftd3_b200.h. */
#pragma once

#ifdef __cplusplus
#define SDFTD3_API_ENTRY extern "C"
#else
#define SDFTD3_API_ENTRY extern
#ifndef SDFTD3_CFFI
#include <stdbool.h>
#endif
#endif
#define SDFTD3_API_CALL
#define SDFTD3_API_SUFFIX__V_0_2
#define SDFTD3_API_SUFFIX__V_0_3
#define SDFTD3_API_SUFFIX__V_0_4
#define SDFTD3_API_SUFFIX__V_0_5
#define SDFTD3_API_SUFFIX__V_1_3
#define SDFTD3_API_SUFFIX__V_1_4
#define SDFTD3_API_SUFFIX__V_1_5
#define SDFTD3_API_SUFFIX__V_1_6

/* Opaque handles (api.f90:87-127) */
typedef struct _dftd3_error* dftd3_error;
typedef struct _dftd3_structure* dftd3_structure;
typedef struct _dftd3_model* dftd3_model;
typedef struct _dftd3_gcp* dftd3_gcp;
typedef struct _dftd3_param* dftd3_param;

#ifndef __cplusplus
#define dftd3_delete(ptr) _Generic((ptr), \
                       dftd3_error: dftd3_delete_error, \
                   dftd3_structure: dftd3_delete_structure, \
                       dftd3_model: dftd3_delete_model, \
                       dftd3_param: dftd3_delete_param, \
                         dftd3_gcp: dftd3_delete_gcp \
                                  )(&ptr)
#endif

/* Version as major*10000 + minor*100 + patch (get_version_api, api.f90:137-146) */
SDFTD3_API_ENTRY int SDFTD3_API_CALL
dftd3_get_version() SDFTD3_API_SUFFIX__V_0_2;

/* Optional feature query; "mpi" is not available (has_feature_api, api.f90:150-164) */
SDFTD3_API_ENTRY bool SDFTD3_API_CALL
dftd3_has_feature(char* /* feature */) SDFTD3_API_SUFFIX__V_1_6;

/* Error handle (new_error_api :168-176, check_error_api :195-213,
 * get_error_api :217-239, delete_error_api :180-191) */
SDFTD3_API_ENTRY dftd3_error SDFTD3_API_CALL
dftd3_new_error() SDFTD3_API_SUFFIX__V_0_2;

SDFTD3_API_ENTRY int SDFTD3_API_CALL
dftd3_check_error(dftd3_error /* error */) SDFTD3_API_SUFFIX__V_0_2;

SDFTD3_API_ENTRY void SDFTD3_API_CALL
dftd3_get_error(dftd3_error /* error */,
                char* /* buffer */,
                const int* /* buffersize */) SDFTD3_API_SUFFIX__V_0_2;

SDFTD3_API_ENTRY void SDFTD3_API_CALL
dftd3_delete_error(dftd3_error* /* error */) SDFTD3_API_SUFFIX__V_0_2;

/* Molecular structure (new_structure_api :243-280, delete_structure_api
 * :284-296, update_structure_api :300-335); positions are wrapped into the
 * central cell and checked for overlapping atoms. */
SDFTD3_API_ENTRY dftd3_structure SDFTD3_API_CALL
dftd3_new_structure(dftd3_error /* error */,
                    const int /* natoms */,
                    const int* /* numbers [natoms] */,
                    const double* /* positions [natoms][3] */,
                    const double* /* lattice [3][3] */,
                    const bool* /* periodic [3] */) SDFTD3_API_SUFFIX__V_0_2;

SDFTD3_API_ENTRY void SDFTD3_API_CALL
dftd3_delete_structure(dftd3_structure* /* mol */) SDFTD3_API_SUFFIX__V_0_2;

SDFTD3_API_ENTRY void SDFTD3_API_CALL
dftd3_update_structure(dftd3_error /* error */,
                       dftd3_structure /* mol */,
                       const double* /* positions [natoms][3] */,
                       const double* /* lattice [3][3] */) SDFTD3_API_SUFFIX__V_0_2;

/* Dispersion model (new_d3_model_api :339-364) */
SDFTD3_API_ENTRY dftd3_model SDFTD3_API_CALL
dftd3_new_d3_model(dftd3_error /* error */,
                   dftd3_structure /* mol */) SDFTD3_API_SUFFIX__V_0_2;

/* Real space cutoffs (set_model_realspace_cutoff :370-392) */
SDFTD3_API_ENTRY void SDFTD3_API_CALL
dftd3_set_model_realspace_cutoff(dftd3_error /* error */,
                                 dftd3_model /* model */,
                                 double /* disp2 */,
                                 double /* disp3 */,
                                 double /* cn */) SDFTD3_API_SUFFIX__V_0_5;

/* Ghost atoms, zero-based indices (set_model_ghost_index :508-537) */
SDFTD3_API_ENTRY void SDFTD3_API_CALL
dftd3_set_model_ghost_index(dftd3_error /* error */,
                            dftd3_model /* model */,
                            const int* /* ghost [nidx] */,
                            int /* nidx */) SDFTD3_API_SUFFIX__V_1_5;

/* Real space cutoffs with smoothing widths (set_model_realspace_cutoff_smooth :395-416) */
SDFTD3_API_ENTRY void SDFTD3_API_CALL
dftd3_set_model_realspace_cutoff_smooth(dftd3_error /* error */,
                                        dftd3_model /* model */,
                                        double /* disp2 */,
                                        double /* disp3 */,
                                        double /* cn */,
                                        double /* width2 */,
                                        double /* width3 */) SDFTD3_API_SUFFIX__V_1_4;

/* Ewald summation (set_model_ewald :426-455): not supported, reports an error */
SDFTD3_API_ENTRY void SDFTD3_API_CALL
dftd3_set_model_ewald(dftd3_error /* error */,
                      dftd3_model /* model */,
                      int /* rank */,
                      double /* tolerance */,
                      double /* kcut */,
                      int /* mesh */) SDFTD3_API_SUFFIX__V_1_6;

/* Externally managed work partition of the pair and triple loops
 * (set_model_work_partition :462-480, partition.f90:80-147) */
SDFTD3_API_ENTRY void SDFTD3_API_CALL
dftd3_set_model_work_partition(dftd3_error /* error */,
                               dftd3_model /* model */,
                               int /* part */,
                               int /* nparts */) SDFTD3_API_SUFFIX__V_1_6;

/* MPI communicator (set_model_mpi_comm :484-506): no MPI build, reports an error */
SDFTD3_API_ENTRY void SDFTD3_API_CALL
dftd3_set_model_mpi_comm(dftd3_error /* error */,
                         dftd3_model /* model */,
                         int /* comm */) SDFTD3_API_SUFFIX__V_1_6;

/* (delete_model_api :541-554) */
SDFTD3_API_ENTRY void SDFTD3_API_CALL
dftd3_delete_model(dftd3_model* /* disp */) SDFTD3_API_SUFFIX__V_0_2;

/* Damping parameters.  Zero (new_zero_damping_api :626-654), rational
 * (new_rational_damping_api :558-586) and the other families below
 * (modified rational and zero, optimized power, CSO, Z; :658-1018) are
 * evaluated on the GPU; the parameter-database loaders (load_*_api,
 * e.g. :590-622) look up the reference's method table. */
SDFTD3_API_ENTRY dftd3_param SDFTD3_API_CALL
dftd3_new_zero_damping(dftd3_error /* error */,
                       double /* s6 */,
                       double /* s8 */,
                       double /* s9 */,
                       double /* rs6 */,
                       double /* rs8 */,
                       double /* alp */) SDFTD3_API_SUFFIX__V_0_4;

SDFTD3_API_ENTRY dftd3_param SDFTD3_API_CALL
dftd3_load_zero_damping(dftd3_error /* error */,
                        char* /* method */,
                        bool /* atm */) SDFTD3_API_SUFFIX__V_0_4;

SDFTD3_API_ENTRY dftd3_param SDFTD3_API_CALL
dftd3_new_rational_damping(dftd3_error /* error */,
                           double /* s6 */,
                           double /* s8 */,
                           double /* s9 */,
                           double /* a1 */,
                           double /* a2 */,
                           double /* alp */) SDFTD3_API_SUFFIX__V_0_4;

SDFTD3_API_ENTRY dftd3_param SDFTD3_API_CALL
dftd3_load_rational_damping(dftd3_error /* error */,
                            char* /* method */,
                            bool /* atm */) SDFTD3_API_SUFFIX__V_0_4;

SDFTD3_API_ENTRY dftd3_param SDFTD3_API_CALL
dftd3_new_mzero_damping(dftd3_error /* error */,
                        double /* s6 */,
                        double /* s8 */,
                        double /* s9 */,
                        double /* rs6 */,
                        double /* rs8 */,
                        double /* alp */,
                        double /* bet */) SDFTD3_API_SUFFIX__V_0_4;

SDFTD3_API_ENTRY dftd3_param SDFTD3_API_CALL
dftd3_load_mzero_damping(dftd3_error /* error */,
                         char* /* method */,
                         bool /* atm */) SDFTD3_API_SUFFIX__V_0_4;

SDFTD3_API_ENTRY dftd3_param SDFTD3_API_CALL
dftd3_new_mrational_damping(dftd3_error /* error */,
                            double /* s6 */,
                            double /* s8 */,
                            double /* s9 */,
                            double /* a1 */,
                            double /* a2 */,
                            double /* alp */) SDFTD3_API_SUFFIX__V_0_4;

SDFTD3_API_ENTRY dftd3_param SDFTD3_API_CALL
dftd3_load_mrational_damping(dftd3_error /* error */,
                             char* /* method */,
                             bool /* atm */) SDFTD3_API_SUFFIX__V_0_4;

SDFTD3_API_ENTRY dftd3_param SDFTD3_API_CALL
dftd3_new_optimizedpower_damping(dftd3_error /* error */,
                                 double /* s6 */,
                                 double /* s8 */,
                                 double /* s9 */,
                                 double /* a1 */,
                                 double /* a2 */,
                                 double /* alp */,
                                 double /* bet */) SDFTD3_API_SUFFIX__V_0_5;

SDFTD3_API_ENTRY dftd3_param SDFTD3_API_CALL
dftd3_load_optimizedpower_damping(dftd3_error /* error */,
                                  char* /* method */,
                                  bool /* atm */) SDFTD3_API_SUFFIX__V_0_5;

SDFTD3_API_ENTRY dftd3_param SDFTD3_API_CALL
dftd3_new_cso_damping(dftd3_error /* error */,
                      double /* s6 */,
                      double /* s9 */,
                      double /* a1 */,
                      double /* a2 */,
                      double /* a3 */,
                      double /* a4 */,
                      double /* alp */) SDFTD3_API_SUFFIX__V_1_3;

SDFTD3_API_ENTRY dftd3_param SDFTD3_API_CALL
dftd3_load_cso_damping(dftd3_error /* error */,
                       char* /* method */,
                       bool /* atm */) SDFTD3_API_SUFFIX__V_1_3;

SDFTD3_API_ENTRY dftd3_param SDFTD3_API_CALL
dftd3_new_z_damping(dftd3_error /* error */,
                    double /* s6 */,
                    double /* s8 */,
                    double /* s9 */,
                    double /* a1 */,
                    double /* alp */) SDFTD3_API_SUFFIX__V_1_4;

SDFTD3_API_ENTRY dftd3_param SDFTD3_API_CALL
dftd3_load_z_damping(dftd3_error /* error */,
                     char* /* method */,
                     bool /* atm */) SDFTD3_API_SUFFIX__V_1_4;

/* (delete_param_api :1022-1034) */
SDFTD3_API_ENTRY void SDFTD3_API_CALL
dftd3_delete_param(dftd3_param* /* param */) SDFTD3_API_SUFFIX__V_0_2;

/* Geometric counter-poise correction: not supported, reports an error */
SDFTD3_API_ENTRY dftd3_gcp SDFTD3_API_CALL
dftd3_load_gcp_param(dftd3_error /* error */,
                     dftd3_structure /* mol */,
                     char* /* method */,
                     char* /* basis */) SDFTD3_API_SUFFIX__V_1_3;

SDFTD3_API_ENTRY void SDFTD3_API_CALL
dftd3_set_gcp_realspace_cutoff(dftd3_error /* error */,
                               dftd3_gcp /* gcp */,
                               double /* bas */,
                               double /* srb */) SDFTD3_API_SUFFIX__V_1_3;

SDFTD3_API_ENTRY void SDFTD3_API_CALL
dftd3_set_gcp_work_partition(dftd3_error /* error */,
                             dftd3_gcp /* gcp */,
                             int /* part */,
                             int /* nparts */) SDFTD3_API_SUFFIX__V_1_6;

SDFTD3_API_ENTRY void SDFTD3_API_CALL
dftd3_set_gcp_mpi_comm(dftd3_error /* error */,
                       dftd3_gcp /* gcp */,
                       int /* comm */) SDFTD3_API_SUFFIX__V_1_6;

SDFTD3_API_ENTRY void SDFTD3_API_CALL
dftd3_delete_gcp(dftd3_gcp* /* gcp */) SDFTD3_API_SUFFIX__V_1_3;

/* Energy, gradient and virial (get_dispersion_api, api.f90:1038-1111).
 * Derivatives are evaluated when gradient or sigma is non-NULL. */
SDFTD3_API_ENTRY void SDFTD3_API_CALL
dftd3_get_dispersion(dftd3_error /* error */,
                     dftd3_structure /* mol */,
                     dftd3_model /* disp */,
                     dftd3_param /* param */,
                     double* /* energy */,
                     double* /* gradient[n][3] */,
                     double* /* sigma[3][3] */) SDFTD3_API_SUFFIX__V_0_2;

/* Pairwise decomposition (get_pairwise_dispersion_api :1180-1233): FP64
 * pair-energy matrices of the two- and three-body terms */
SDFTD3_API_ENTRY void SDFTD3_API_CALL
dftd3_get_pairwise_dispersion(dftd3_error /* error */,
                              dftd3_structure /* mol */,
                              dftd3_model /* disp */,
                              dftd3_param /* param */,
                              double* /* pair_energy2[n][n] */,
                              double* /* pair_energy3[n][n] */) SDFTD3_API_SUFFIX__V_0_5;

/* Analytical Hessian (get_dispersion_hessian_api :1115-1176): FP64 energy
 * and Hessian of one structure */
SDFTD3_API_ENTRY void SDFTD3_API_CALL
dftd3_get_dispersion_hessian(dftd3_error /* error */,
                             dftd3_structure /* mol */,
                             dftd3_model /* disp */,
                             dftd3_param /* param */,
                             double* /* energy */,
                             double* /* hessian[3*n][3*n] */) SDFTD3_API_SUFFIX__V_1_6;

SDFTD3_API_ENTRY void SDFTD3_API_CALL
dftd3_get_counterpoise(dftd3_error /* error */,
                       dftd3_structure /* mol */,
                       dftd3_gcp /* gcp */,
                       double* /* energy */,
                       double* /* gradient[n][3] */,
                       double* /* sigma[3][3] */) SDFTD3_API_SUFFIX__V_1_3;

SDFTD3_API_ENTRY void SDFTD3_API_CALL
dftd3_get_counterpoise_hessian(dftd3_error /* error */,
                               dftd3_structure /* mol */,
                               dftd3_gcp /* gcp */,
                               double* /* energy */,
                               double* /* hessian[3*n][3*n] */) SDFTD3_API_SUFFIX__V_1_6;
