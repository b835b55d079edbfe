/* D3 model parameter tables (generated data, see gen_tables.py) and the
 * unit constants the model setup uses.
 *
 * Element limits follow the reference: reference C6 data and van-der-Waals
 * radii exist for Z <= 103 (reference.f90:27, data/vdwrad.f90:36), r4/r2 and
 * covalent radii for Z <= 118 (data/r4r2.f90:34). */
#pragma once

#ifdef __cplusplus
extern "C" {
#endif

#define D3_MAX_ELEM 103
#define D3_MAX_ELEM_R4R2 118
#define D3_MAX_REF 7

extern const unsigned char d3_nref[D3_MAX_ELEM];
extern const double d3_refcn[D3_MAX_ELEM * D3_MAX_REF];
extern const double d3_r4_over_r2[D3_MAX_ELEM_R4R2];
extern const double d3_rcov_aa[D3_MAX_ELEM_R4R2];
extern const double d3_vdwrad_aa[D3_MAX_ELEM * (D3_MAX_ELEM + 1) / 2];
extern const double d3_c6ab[D3_MAX_REF * D3_MAX_REF * D3_MAX_ELEM * (D3_MAX_ELEM + 1) / 2];

/* Bohr radius in Angstrom (CODATA 2018, the value mctc-lib's unit module
 * carries) and its inverse, the Angstrom-to-Bohr factor. */
#define D3_AUTOAA 0.52917721090380
#define D3_AATOAU (1.0 / D3_AUTOAA)

#ifdef __cplusplus
}
#endif
