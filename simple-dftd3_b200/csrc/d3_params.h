/* Damping parameter database (d3_params.c, generated by gen_params.py from
 * the reference's src/dftd3/param.f90). */
#pragma once

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    const char* name;   /* normalised method name: '-' removed, lower case */
    int id;             /* method id */
} d3_method_alias;

typedef struct {
    int id;             /* method id */
    double v[9];        /* s6, s8, s9, rs6, rs8, a1, a2, alp, bet */
} d3_param_record;

extern const d3_method_alias d3_method_aliases[];
extern const int d3_n_method_aliases;
extern const d3_param_record d3_rational_params[];
extern const int d3_n_rational_params;
extern const d3_param_record d3_zero_params[];
extern const int d3_n_zero_params;
extern const d3_param_record d3_mrational_params[];
extern const int d3_n_mrational_params;
extern const d3_param_record d3_mzero_params[];
extern const int d3_n_mzero_params;
extern const d3_param_record d3_optimizedpower_params[];
extern const int d3_n_optimizedpower_params;
extern const d3_param_record d3_cso_params[];   /* a3, a4 in the rs6, rs8 slots */
extern const int d3_n_cso_params;
extern const d3_param_record d3_z_params[];
extern const int d3_n_z_params;

#ifdef __cplusplus
}
#endif
