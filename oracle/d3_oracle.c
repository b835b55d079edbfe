/* FP64 CPU oracle for the D3 dispersion hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use
 * this file, as the checker.  It is a loop-for-loop restatement of the
 * reference Fortran (s-dftd3 v1.6.0); every function names the file:line it
 * follows.  Loop orders, expression orders and the OpenMP thread-private
 * accumulation follow the reference so the results agree to rounding.
 *
 * Parity pins: the tests compare this oracle with the reference's golden
 * vectors (the JSON files in tests/golden, generated from the reference's test files by
 * tests/golden/make_golden.py). */
#include "d3_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#include "../simple-dftd3_b200/csrc/d3_tables.h"

#define EPS DBL_EPSILON
#define KCN 16.0                 /* ncoord.f90:31 */
#define WF 4.0                   /* model.f90:80 */
#define RS9 (4.0 / 3.0)          /* rational.f90:73, zero.f90:77 */

/* ---------------------------------------------------------------- model -- */

typedef struct {
    int nid, mref;
    int *id;          /* [nat] species index */
    int *num;         /* [nid] atomic number */
    int *ref;         /* [nid] */
    double *rcov;     /* [nid] */
    double *r4r2;     /* [nid] */
    double *rvdw;     /* [nid][nid] */
    double *cn;       /* [nid][mref], cn[isp*mref + iref] */
    double *c6;       /* c6(iref, jref, isp, jsp) at ((isp*nid + jsp)*mref + iref)*mref + jref */
    int *ghost;       /* [nat] */
} model_t;

double oracle_covalent_radius(int z)
{
    /* mctc-lib get_covalent_rad: 4/3 scaled D3 covalent radius in Bohr */
    if (z < 1 || z > D3_MAX_ELEM_R4R2) return 0.0;
    return 4.0 / 3.0 * (D3_AATOAU * d3_rcov_aa[z - 1]);
}

double oracle_r4r2(int z)
{
    /* data/r4r2.f90:69-70, 91-105 */
    if (z < 1 || z > D3_MAX_ELEM_R4R2) return 0.0;
    return sqrt(0.5 * (d3_r4_over_r2[z - 1] * sqrt((double)z)));
}

static double get_vdw_rad(int z1, int z2)
{
    /* data/vdwrad.f90:1163-1197 (both inside the table for Z <= 103) */
    int ic = z1 > z2 ? (z2 - 1) + z1 * (z1 - 1) / 2 : (z1 - 1) + z2 * (z2 - 1) / 2;
    return D3_AATOAU * d3_vdwrad_aa[ic];
}

static double get_c6(int iref, int jref, int ati, int atj)
{
    /* reference.f90:160-171, 0-based reference indices, 1-based Z */
    int ic;
    if (ati > atj) {
        ic = (atj - 1) + ati * (ati - 1) / 2;
        return d3_c6ab[ic * 49 + jref * 7 + iref];
    }
    ic = (ati - 1) + atj * (atj - 1) / 2;
    return d3_c6ab[ic * 49 + iref * 7 + jref];
}

static void model_free(model_t *m)
{
    free(m->id); free(m->num); free(m->ref); free(m->rcov); free(m->r4r2);
    free(m->rvdw); free(m->cn); free(m->c6); free(m->ghost);
}

static int model_new(model_t *m, int nat, const int *numbers, const int *ghost)
{
    /* species by first occurrence (mctc-lib structure constructor), then
     * new_d3_model (model.f90:87-181) */
    memset(m, 0, sizeof(*m));
    m->id = malloc(sizeof(int) * (nat > 0 ? nat : 1));
    m->num = malloc(sizeof(int) * (nat > 0 ? nat : 1));
    for (int i = 0; i < nat; i++) {
        int z = numbers[i], s;
        if (z < 1 || z > D3_MAX_ELEM) { free(m->id); free(m->num); return 1; }
        for (s = 0; s < m->nid; s++) if (m->num[s] == z) break;
        if (s == m->nid) m->num[m->nid++] = z;
        m->id[i] = s;
    }
    int nid = m->nid;
    m->ref = malloc(sizeof(int) * nid);
    m->mref = 0;
    for (int s = 0; s < nid; s++) {
        m->ref[s] = d3_nref[m->num[s] - 1];
        if (m->ref[s] > m->mref) m->mref = m->ref[s];
    }
    int mref = m->mref;
    m->rcov = malloc(sizeof(double) * nid);
    m->r4r2 = malloc(sizeof(double) * nid);
    for (int s = 0; s < nid; s++) {
        m->rcov[s] = oracle_covalent_radius(m->num[s]);
        m->r4r2[s] = oracle_r4r2(m->num[s]);
    }
    m->rvdw = malloc(sizeof(double) * nid * nid);
    for (int is = 0; is < nid; is++)
        for (int js = 0; js <= is; js++) {
            double r = get_vdw_rad(m->num[js], m->num[is]);
            m->rvdw[js * nid + is] = r;
            m->rvdw[is * nid + js] = r;
        }
    m->cn = calloc((size_t)mref * nid, sizeof(double));
    for (int s = 0; s < nid; s++)
        for (int r = 0; r < m->ref[s]; r++)
            m->cn[s * mref + r] = d3_refcn[(m->num[s] - 1) * 7 + r];
    m->c6 = calloc((size_t)mref * mref * nid * nid, sizeof(double));
#define MC6(ir, jr, is, js) m->c6[(((size_t)(is) * nid + (js)) * mref + (ir)) * mref + (jr)]
    for (int is = 0; is < nid; is++)
        for (int js = 0; js <= is; js++)
            for (int ir = 0; ir < m->ref[is]; ir++)
                for (int jr = 0; jr < m->ref[js]; jr++) {
                    MC6(jr, ir, js, is) = get_c6(jr, ir, m->num[js], m->num[is]);
                    MC6(ir, jr, is, js) = MC6(jr, ir, js, is);
                }
    m->ghost = calloc(nat > 0 ? nat : 1, sizeof(int));
    if (ghost)
        for (int i = 0; i < nat; i++) m->ghost[i] = ghost[i] != 0;
    return 0;
}

/* --------------------------------------------------------------- cutoff -- */

static void crossproduct(const double *a, const double *b, double *c)
{
    /* cutoff.f90:229-238 */
    double x = a[1] * b[2] - b[1] * a[2];
    double y = a[2] * b[0] - b[2] * a[0];
    double z = a[0] * b[1] - b[0] * a[1];
    c[0] = x; c[1] = y; c[2] = z;
}

/* lat[k][c]: column k of the Fortran lat(3,3), i.e. vector k */
static void get_translations(const double lat[3][3], double rthr, int rep[3])
{
    /* cutoff.f90:204-227 */
    double norm[3][3];
    crossproduct(lat[1], lat[2], norm[0]);
    crossproduct(lat[2], lat[0], norm[1]);
    crossproduct(lat[0], lat[1], norm[2]);
    for (int k = 0; k < 3; k++) {
        double n2 = sqrt(norm[k][0] * norm[k][0] + norm[k][1] * norm[k][1] + norm[k][2] * norm[k][2]);
        for (int c = 0; c < 3; c++) norm[k][c] = norm[k][c] / n2;
    }
    for (int k = 0; k < 3; k++) {
        double cs = norm[k][0] * lat[k][0] + norm[k][1] * lat[k][1] + norm[k][2] * lat[k][2];
        rep[k] = (int)ceil(fabs(rthr / cs));
    }
}

int oracle_lattice_points(const double *lattice, const int *periodic, double rthr,
                          double *trans, int cap)
{
    /* get_lattice_points, cutoff.f90:140-186 */
    int np = (periodic[0] != 0) + (periodic[1] != 0) + (periodic[2] != 0);
    double lat[3][3];
    int rep[3] = {0, 0, 0};
    if (np == 0) {
        if (trans && cap >= 1) trans[0] = trans[1] = trans[2] = 0.0;
        return 1;
    }
    for (int k = 0; k < 3; k++)
        for (int c = 0; c < 3; c++) lat[k][c] = lattice[k * 3 + c];
    if (np == 3) {
        get_translations(lat, rthr, rep);
    } else if (np == 1) {
        for (int k = 0; k < 3; k++) {
            double v = sqrt(lat[k][0] * lat[k][0] + lat[k][1] * lat[k][1] + lat[k][2] * lat[k][2]);
            rep[k] = periodic[k] ? (int)ceil(rthr / v) : 0;
        }
    } else {
        /* get_normals, then norms(i, :) = lat(i, :) where periodic(i) */
        double norms[3][3];
        for (int k = 0; k < 3; k++)
            crossproduct(lat[(k + 1) % 3], lat[(k + 2) % 3], norms[k]);
        for (int k = 0; k < 3; k++)
            for (int c = 0; c < 3; c++)
                if (periodic[c]) norms[k][c] = lat[k][c];
        get_translations(norms, rthr, rep);
        for (int k = 0; k < 3; k++) if (!periodic[k]) rep[k] = 0;
    }
    int n = (2 * rep[0] + 1) * (2 * rep[1] + 1) * (2 * rep[2] + 1);
    if (trans && cap >= n) {
        int itr = 0;
        for (int ix = -rep[0]; ix <= rep[0]; ix++)
            for (int iy = -rep[1]; iy <= rep[1]; iy++)
                for (int iz = -rep[2]; iz <= rep[2]; iz++, itr++)
                    for (int c = 0; c < 3; c++)
                        trans[itr * 3 + c] = lat[0][c] * ix + lat[1][c] * iy + lat[2][c] * iz;
    }
    return n;
}

static double *lattice_points(const double *lattice, const int *periodic, double rthr, int *ntr)
{
    int n = oracle_lattice_points(lattice, periodic, rthr, NULL, 0);
    double *t = malloc(sizeof(double) * 3 * n);
    oracle_lattice_points(lattice, periodic, rthr, t, n);
    *ntr = n;
    return t;
}

static void smooth_cutoff(double r, double cutoff, double width, double *sw, double *dswdr)
{
    /* cutoff.f90:73-99 */
    if (width <= 0.0 || width >= cutoff) {
        *sw = 1.0; *dswdr = 0.0;
    } else {
        double inner = cutoff - width;
        if (r <= inner) { *sw = 1.0; *dswdr = 0.0; }
        else if (r >= cutoff) { *sw = 0.0; *dswdr = 0.0; }
        else {
            double x = (cutoff - r) / width;
            *sw = x * x * x * (10.0 + x * (-15.0 + 6.0 * x));
            *dswdr = -30.0 * x * x * (1.0 - x) * (1.0 - x) / width;
        }
    }
}

/* ------------------------------------------------------------ partition -- */

static int owns_pair(int part, int nparts, int i, int j)
{
    /* partition.f90:127-147 with 0-based i >= j */
    if (nparts <= 1) return 1;
    long long idx = (long long)i * (i + 1) / 2 + j;
    return idx % nparts == part;
}

/* ------------------------------------------------------------------ wrap -- */

static void matinv_3x3(const double a[3][3], double inv[3][3])
{
    /* inverse by cofactors (mctc-lib matinv_3x3); a[r][c] is row r, col c */
    double det = a[0][0] * a[1][1] * a[2][2] - a[0][0] * a[1][2] * a[2][1]
               - a[0][1] * a[1][0] * a[2][2] + a[0][1] * a[1][2] * a[2][0]
               + a[0][2] * a[1][0] * a[2][1] - a[0][2] * a[1][1] * a[2][0];
    double d = 1.0 / det;
    inv[0][0] = +d * (a[1][1] * a[2][2] - a[1][2] * a[2][1]);
    inv[1][0] = -d * (a[1][0] * a[2][2] - a[1][2] * a[2][0]);
    inv[2][0] = +d * (a[1][0] * a[2][1] - a[1][1] * a[2][0]);
    inv[0][1] = -d * (a[0][1] * a[2][2] - a[0][2] * a[2][1]);
    inv[1][1] = +d * (a[0][0] * a[2][2] - a[0][2] * a[2][0]);
    inv[2][1] = -d * (a[0][0] * a[2][1] - a[0][1] * a[2][0]);
    inv[0][2] = +d * (a[0][1] * a[1][2] - a[0][2] * a[1][1]);
    inv[1][2] = -d * (a[0][0] * a[1][2] - a[0][2] * a[1][0]);
    inv[2][2] = +d * (a[0][0] * a[1][1] - a[0][1] * a[1][0]);
}

static double shift_back_abc(double in)
{
    /* utils.f90:48-64 */
    const double eps = 1.0e-14;
    double out = in;
    if (in < (0.0 - eps)) out = in + ceil(-in);
    if (in > (1.0 + eps)) out = in - floor(in);
    if (fabs(in - 1.0) < eps) out = in - 1.0;
    return out;
}

void oracle_wrap_to_central_cell(int nat, double *xyz, const double *lattice, const int *periodic)
{
    /* utils.f90:29-44: matrix M has the lattice vectors as columns */
    if (!(periodic[0] || periodic[1] || periodic[2])) return;
    double m[3][3], inv[3][3];
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) m[r][c] = lattice[c * 3 + r];
    matinv_3x3(m, inv);
    for (int i = 0; i < nat; i++) {
        double *x = xyz + 3 * i, f[3];
        for (int r = 0; r < 3; r++)
            f[r] = shift_back_abc(inv[r][0] * x[0] + inv[r][1] * x[1] + inv[r][2] * x[2]);
        for (int r = 0; r < 3; r++)
            x[r] = m[r][0] * f[0] + m[r][1] * f[1] + m[r][2] * f[2];
    }
}

/* --------------------------------------------------------------- ncoord -- */

static void partitioned_cn(int nat, const double *xyz, const int *id, const double *rcov,
                           const double *trans, int ntr, double cutoff, double *cn, int part, int nparts)
{
    /* get_partitioned_coordination_number, ncoord.f90:86-144; nparts = 1 is
     * the complete work */
    double cutoff2 = cutoff * cutoff;
    for (int i = 0; i < nat; i++) cn[i] = 0.0;
#pragma omp parallel
    {
        double *loc = calloc(nat, sizeof(double));
#pragma omp for schedule(dynamic, 1)
        for (int i = 0; i < nat; i++) {
            int izp = id[i];
            for (int j = 0; j <= i; j++) {
                if (!owns_pair(part, nparts, i, j)) continue;
                int jzp = id[j];
                double rc = rcov[izp] + rcov[jzp];
                for (int t = 0; t < ntr; t++) {
                    double v0 = xyz[3 * i + 0] - (xyz[3 * j + 0] + trans[3 * t + 0]);
                    double v1 = xyz[3 * i + 1] - (xyz[3 * j + 1] + trans[3 * t + 1]);
                    double v2 = xyz[3 * i + 2] - (xyz[3 * j + 2] + trans[3 * t + 2]);
                    double r2 = v0 * v0 + v1 * v1 + v2 * v2;
                    if (r2 > cutoff2 || r2 < 1.0e-12) continue;
                    double r1 = sqrt(r2);
                    double countf = 1.0 / (1.0 + exp(-KCN * (rc / r1 - 1.0)));
                    loc[i] += countf;
                    if (i != j) loc[j] += countf;
                }
            }
        }
#pragma omp critical(oracle_cn)
        for (int i = 0; i < nat; i++) cn[i] += loc[i];
        free(loc);
    }
}

static void add_cn_derivs(int nat, const double *xyz, const int *id, const double *rcov,
                          const double *trans, int ntr, double cutoff, const double *dEdcn,
                          double *gradient, double *sigma, int part, int nparts)
{
    /* add_coordination_number_derivs, ncoord.f90:152-228; nparts = 1 is the
     * complete work */
    double cutoff2 = cutoff * cutoff;
#pragma omp parallel
    {
        double *gl = calloc(3 * (size_t)nat, sizeof(double));
        double sl[9] = {0};
#pragma omp for schedule(dynamic, 1)
        for (int i = 0; i < nat; i++) {
            int izp = id[i];
            for (int j = 0; j <= i; j++) {
                if (!owns_pair(part, nparts, i, j)) continue;
                int jzp = id[j];
                double rc = rcov[izp] + rcov[jzp];
                for (int t = 0; t < ntr; t++) {
                    double v[3];
                    for (int c = 0; c < 3; c++)
                        v[c] = xyz[3 * i + c] - (xyz[3 * j + c] + trans[3 * t + c]);
                    double r2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
                    if (r2 > cutoff2 || r2 < 1.0e-12) continue;
                    double r1 = sqrt(r2);
                    double expterm = exp(-KCN * (rc / r1 - 1.0));
                    double cf = 1.0 / (1.0 + expterm);
                    double dcf = -cf * (1.0 - cf) * KCN * rc / r2;
                    double cd[3];
                    for (int c = 0; c < 3; c++) cd[c] = dcf * v[c] / r1;
                    double de = dEdcn[i] + dEdcn[j];
                    for (int c = 0; c < 3; c++) {
                        gl[3 * i + c] += cd[c] * de;
                        gl[3 * j + c] -= cd[c] * de;
                    }
                    double w = dEdcn[i] + (j != i ? dEdcn[j] : 0.0);
                    for (int a = 0; a < 3; a++)
                        for (int b = 0; b < 3; b++) sl[a + 3 * b] += cd[a] * v[b] * w;
                }
            }
        }
#pragma omp critical(oracle_cnd)
        {
            for (int k = 0; k < 3 * nat; k++) gradient[k] += gl[k];
            for (int k = 0; k < 9; k++) sigma[k] += sl[k];
        }
        free(gl);
    }
}

int oracle_coordination_number(int nat, const int *numbers, const double *xyz,
                               const double *lattice, const int *periodic, double cutoff, double *cn)
{
    model_t m;
    if (model_new(&m, nat, numbers, NULL)) return 1;
    int ntr;
    double zero[9] = {0};
    double *trans = lattice_points(lattice ? lattice : zero, periodic, cutoff, &ntr);
    partitioned_cn(nat, xyz, m.id, m.rcov, trans, ntr, cutoff, cn, 0, 1);
    free(trans);
    model_free(&m);
    return 0;
}

/* ---------------------------------------------------------------- model -- */

static int is_exceptional(double v) { return isnan(v) || fabs(v) > DBL_MAX; }

static void weight_references(const model_t *m, int nat, const double *cn,
                              double *gwvec, double *gwdcn)
{
    /* model.f90:201-324 (first-derivative and energy-only branches), with
     * gwvec(iref, iat) at [iat*mref + iref] */
    int mref = m->mref;
    double wf2 = 2 * WF;
    for (int k = 0; k < nat * mref; k++) {
        gwvec[k] = 0.0;
        if (gwdcn) gwdcn[k] = 0.0;
    }
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nat; i++) {
        int izp = m->id[i];
        int nref = m->ref[izp];
        const double *cnref = m->cn + izp * mref;
        double gwt[D3_MAX_REF];
        double norm = 0.0, dnorm = 0.0;
        for (int r = 0; r < nref; r++) {
            double gw = exp(-WF * (cn[i] - cnref[r]) * (cn[i] - cnref[r]));
            gwt[r] = gw;
            double dcn = cnref[r] - cn[i];
            norm = norm + gw;
            dnorm = dnorm + wf2 * dcn * gw;
        }
        norm = 1.0 / norm;
        double maxcn = cnref[0];
        for (int r = 1; r < nref; r++) if (cnref[r] > maxcn) maxcn = cnref[r];
        for (int r = 0; r < nref; r++) {
            double expw = gwt[r];
            double dcn = cnref[r] - cn[i];
            double expd = wf2 * dcn * expw;
            double gwk = expw * norm;
            if (is_exceptional(gwk)) gwk = (maxcn == cnref[r]) ? 1.0 : 0.0;
            gwvec[i * mref + r] = gwk;
            if (gwdcn) {
                double dgwk = expd * norm - expw * dnorm * (norm * norm);
                if (is_exceptional(dgwk)) dgwk = 0.0;
                gwdcn[i * mref + r] = dgwk;
            }
        }
    }
}

int oracle_weight_references(int nat, const int *numbers, const double *cn,
                             int *mref_out, double *gwvec, double *gwdcn)
{
    model_t m;
    if (model_new(&m, nat, numbers, NULL)) return 1;
    *mref_out = m.mref;
    if (gwvec) weight_references(&m, nat, cn, gwvec, gwdcn);
    model_free(&m);
    return 0;
}

static void get_atomic_c6(const model_t *m, int nat, const double *gwvec, const double *gwdcn,
                          double *c6, double *dc6dcn, int part, int nparts)
{
    /* model.f90:340-491 (first-derivative and energy-only branches);
     * c6(iat, jat) at [iat*nat + jat], dc6dcn(iat, jat) = dC6_ij/dCN_i */
    int mref = m->mref, nid = m->nid;
    memset(c6, 0, sizeof(double) * (size_t)nat * nat);
    if (dc6dcn) memset(dc6dcn, 0, sizeof(double) * (size_t)nat * nat);
#pragma omp parallel for schedule(dynamic, 1)
    for (int i = 0; i < nat; i++) {
        if (m->ghost[i]) continue;
        int izp = m->id[i];
        for (int j = 0; j <= i; j++) {
            if (m->ghost[j]) continue;
            if (!owns_pair(part, nparts, i, j)) continue;
            int jzp = m->id[j];
            double dc6 = 0.0, dci = 0.0, dcj = 0.0;
            for (int ir = 0; ir < m->ref[izp]; ir++)
                for (int jr = 0; jr < m->ref[jzp]; jr++) {
                    double refc6 = m->c6[(((size_t)izp * nid + jzp) * mref + ir) * mref + jr];
                    dc6 = dc6 + gwvec[i * mref + ir] * gwvec[j * mref + jr] * refc6;
                    if (dc6dcn) {
                        dci = dci + gwdcn[i * mref + ir] * gwvec[j * mref + jr] * refc6;
                        dcj = dcj + gwvec[i * mref + ir] * gwdcn[j * mref + jr] * refc6;
                    }
                }
            c6[(size_t)i * nat + j] = dc6;
            c6[(size_t)j * nat + i] = dc6;
            if (dc6dcn) {
                dc6dcn[(size_t)i * nat + j] = dci;
                dc6dcn[(size_t)j * nat + i] = dcj;
            }
        }
    }
}

/* -------------------------------------------------------------- two-body -- */

static void dispersion2(const model_t *m, const oracle_param *p, int nat, const double *xyz,
                        const double *trans, int ntr, double cutoff, double width,
                        const double *c6, const double *dc6dcn, double *energy,
                        double *dEdcn, double *gradient, double *sigma, int part, int nparts)
{
    /* rational.f90:220-514, zero.f90:306-553, mzero.f90:196-553,
     * optimizedpower.f90:179-483, cso.f90:177-476 and z.f90:176-466;
     * derivatives when dEdcn != NULL */
    if (p->damping == ORACLE_CSO) {
        if (fabs(p->s6) < EPS && fabs(p->a1) < EPS) return;      /* cso.f90:223 */
    } else if (fabs(p->s6) < EPS && fabs(p->s8) < EPS) {
        return;
    }
    double cutoff2 = cutoff * cutoff;
    int grad = dEdcn != NULL;
    double alp6 = p->alp, alp8 = p->alp + 2.0;
#pragma omp parallel
    {
        double *el = calloc(nat, sizeof(double));
        double *dl = grad ? calloc(nat, sizeof(double)) : NULL;
        double *gl = grad ? calloc(3 * (size_t)nat, sizeof(double)) : NULL;
        double sl[9] = {0};
#pragma omp for schedule(dynamic, 1)
        for (int i = 0; i < nat; i++) {
            int izp = m->id[i];
            for (int j = 0; j <= i; j++) {
                if (!owns_pair(part, nparts, i, j)) continue;
                int jzp = m->id[j];
                double rrij = 3 * m->r4r2[izp] * m->r4r2[jzp];
                double c6ij = c6[(size_t)j * nat + i];
                double r0ij = 0, r0ij6 = 0, r0ij8 = 0, rs6r0 = 0, rs8r0 = 0;
                double irs6r0 = 0, irs8r0 = 0, betr0 = 0, betr02rs6 = 0, betr02rs8 = 0;
                double abr0ij6 = 0, abr0ij8 = 0, d6_6 = 0, a2r0ij = 0, zr0c6 = 0;
                switch (p->damping) {
                case ORACLE_RATIONAL: {
                    r0ij = p->a1 * sqrt(rrij) + p->a2;
                    double r0ij2 = r0ij * r0ij;
                    r0ij6 = r0ij2 * r0ij2 * r0ij2;
                    r0ij8 = r0ij6 * r0ij2;
                    break;
                }
                case ORACLE_ZERO:
                    r0ij = m->rvdw[jzp * m->nid + izp];
                    rs6r0 = p->rs6 * r0ij;
                    rs8r0 = p->rs8 * r0ij;
                    break;
                case ORACLE_MZERO:            /* mzero.f90:441-447 */
                    r0ij = m->rvdw[jzp * m->nid + izp];
                    irs6r0 = 1.0 / (p->rs6 * r0ij);
                    irs8r0 = 1.0 / (p->rs8 * r0ij);
                    betr0 = p->bet * r0ij;
                    betr02rs6 = p->rs6 * p->bet * r0ij * r0ij;
                    betr02rs8 = p->rs8 * p->bet * r0ij * r0ij;
                    break;
                case ORACLE_OPTIMIZEDPOWER: { /* optimizedpower.f90:421-429 */
                    r0ij = p->a1 * sqrt(rrij) + p->a2;
                    double r0ij2 = r0ij * r0ij;
                    r0ij6 = r0ij2 * r0ij2 * r0ij2;
                    r0ij8 = r0ij6 * r0ij2;
                    double ab = pow(r0ij, p->bet);
                    abr0ij6 = ab * r0ij6;
                    abr0ij8 = ab * r0ij8;
                    break;
                }
                case ORACLE_CSO:              /* cso.f90:421-426, a3 = rs6, a4 = rs8 */
                    r0ij = sqrt(rrij);
                    d6_6 = pow(p->rs6 * r0ij + p->rs8, 6);
                    a2r0ij = p->a2 * r0ij;
                    break;
                default:                      /* Z, z.f90:412-414: species indices from 1 */
                    r0ij = p->a1 / (double)((izp + 1) + (jzp + 1));
                    zr0c6 = r0ij * c6ij;
                    break;
                }
                for (int t = 0; t < ntr; t++) {
                    double v[3];
                    for (int c = 0; c < 3; c++)
                        v[c] = xyz[3 * i + c] - (xyz[3 * j + c] + trans[3 * t + c]);
                    double r2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
                    if (r2 > cutoff2 || r2 < EPS) continue;
                    double r1 = sqrt(r2);
                    double sw, dswdr;
                    smooth_cutoff(r1, cutoff, width, &sw, &dswdr);
                    double edisp0, gdisp0;
                    /* dE/dC6 of the pair is -sw * cdisp0 for every family; only
                     * Z damping has cdisp0 != edisp0 (z.f90:431) */
                    double cdisp0 = 0.0;
                    switch (p->damping) {
                    case ORACLE_RATIONAL: {
                        double r4 = r2 * r2;
                        double t6 = 1.0 / (r4 * r2 + r0ij6);
                        double t8 = 1.0 / (r4 * r4 + r0ij8);
                        double d6 = -6 * r4 * t6 * t6;
                        double d8 = -8 * r4 * r2 * t8 * t8;
                        edisp0 = p->s6 * t6 + p->s8 * rrij * t8;
                        gdisp0 = p->s6 * d6 + p->s8 * rrij * d8;
                        break;
                    }
                    case ORACLE_ZERO: {
                        double r6 = r2 * r2 * r2;
                        double r8 = r6 * r2;
                        double t6 = pow(rs6r0 / r1, alp6);
                        double t8 = pow(rs8r0 / r1, alp8);
                        double f6 = 1.0 / (1.0 + 6.0 * t6);
                        double f8 = 1.0 / (1.0 + 6.0 * t8);
                        double d6 = -6.0 * f6 / r2 + 6.0 * alp6 * t6 * (f6 * f6) / r2;
                        double d8 = -8.0 * f8 / r2 + 6.0 * alp8 * t8 * (f8 * f8) / r2;
                        edisp0 = p->s6 * f6 / r6 + p->s8 * rrij * f8 / r8;
                        gdisp0 = p->s6 * d6 / r6 + p->s8 * rrij * d8 / r8;
                        break;
                    }
                    case ORACLE_MZERO: {      /* mzero.f90:456-472 */
                        double r6 = r2 * r2 * r2;
                        double r8 = r6 * r2;
                        double t6 = pow(r1 * irs6r0 + betr0, -alp6);
                        double t8 = pow(r1 * irs8r0 + betr0, -alp8);
                        double f6 = 1.0 / (1.0 + 6.0 * t6);
                        double f8 = 1.0 / (1.0 + 6.0 * t8);
                        double d6 = -6.0 * f6 / r2 + 6.0 * alp6 * t6 * (f6 * f6) / (r2 + betr02rs6 * r1);
                        double d8 = -8.0 * f8 / r2 + 6.0 * alp8 * t8 * (f8 * f8) / (r2 + betr02rs8 * r1);
                        edisp0 = p->s6 * f6 / r6 + p->s8 * rrij * f8 / r8;
                        gdisp0 = p->s6 * d6 / r6 + p->s8 * rrij * d8 / r8;
                        break;
                    }
                    case ORACLE_OPTIMIZEDPOWER: { /* optimizedpower.f90:438-448 */
                        double rb = pow(r2, p->bet * 0.5);
                        double r4 = r2 * r2;
                        double t6 = rb / (rb * r4 * r2 + abr0ij6);
                        double t8 = rb / (rb * r4 * r4 + abr0ij8);
                        double d6 = -6 * r4 * t6 * t6 + p->bet * abr0ij6 * t6 * t6 / (rb * r2);
                        double d8 = -8 * r4 * r2 * t8 * t8 + p->bet * abr0ij8 * t8 * t8 / (rb * r2);
                        edisp0 = p->s6 * t6 + p->s8 * rrij * t8;
                        gdisp0 = p->s6 * d6 + p->s8 * rrij * d8;
                        break;
                    }
                    case ORACLE_CSO: {        /* cso.f90:434-446 */
                        double ef = exp(r1 - a2r0ij);
                        double sf = 1.0 / (1.0 + ef);
                        double sig = p->s6 + p->a1 * sf;
                        double r4 = r2 * r2;
                        double t6 = 1.0 / (r4 * r2 + d6_6);
                        double dsig = -p->a1 * sf * (1.0 - sf) / r1;
                        double dt6 = -6 * r4 * t6 * t6;
                        edisp0 = sig * t6;
                        gdisp0 = dsig * t6 + sig * dt6;
                        break;
                    }
                    default: {                /* Z, z.f90:421-431 */
                        double r4 = r2 * r2;
                        double t6 = 1.0 / (r4 * r2 + zr0c6);
                        double t8 = 1.0 / (r4 * r4 + zr0c6 * rrij);
                        double d6 = -6 * r4 * t6 * t6;
                        double d8 = -8 * r4 * r2 * t8 * t8;
                        edisp0 = p->s6 * t6 + p->s8 * rrij * t8;
                        gdisp0 = p->s6 * d6 + p->s8 * rrij * d8;
                        cdisp0 = p->s6 * r4 * r2 * t6 * t6 + p->s8 * rrij * r4 * r4 * t8 * t8;
                        break;
                    }
                    }
                    if (p->damping != ORACLE_Z) cdisp0 = edisp0;
                    double edisp = sw * edisp0;
                    double dE = -c6ij * edisp * 0.5;
                    el[i] += dE;
                    if (i != j) el[j] += dE;
                    if (!grad) continue;
                    double gdisp = sw * gdisp0 + dswdr * edisp0 / r1;
                    double dG[3];
                    for (int c = 0; c < 3; c++) dG[c] = -c6ij * gdisp * v[c];
                    double dS[9];
                    for (int a = 0; a < 3; a++)
                        for (int b = 0; b < 3; b++) dS[a + 3 * b] = dG[a] * v[b] * 0.5;
                    double cdisp = sw * cdisp0;
                    dl[i] -= dc6dcn[(size_t)i * nat + j] * cdisp;
                    for (int k = 0; k < 9; k++) sl[k] += dS[k];
                    if (i != j) {
                        dl[j] -= dc6dcn[(size_t)j * nat + i] * cdisp;
                        for (int c = 0; c < 3; c++) {
                            gl[3 * i + c] += dG[c];
                            gl[3 * j + c] -= dG[c];
                        }
                        for (int k = 0; k < 9; k++) sl[k] += dS[k];
                    }
                }
            }
        }
#pragma omp critical(oracle_disp2)
        {
            for (int i = 0; i < nat; i++) energy[i] += el[i];
            if (grad) {
                for (int i = 0; i < nat; i++) dEdcn[i] += dl[i];
                for (int k = 0; k < 3 * nat; k++) gradient[k] += gl[k];
                for (int k = 0; k < 9; k++) sigma[k] += sl[k];
            }
        }
        free(el); free(dl); free(gl);
    }
}

/* ------------------------------------------------------------ three-body -- */

static double triple_scale(int ii, int jj, int kk)
{
    /* atm.f90:954-980 */
    if (ii == jj) return ii == kk ? 1.0 / 6.0 : 0.5;
    return (ii != kk && jj != kk) ? 1.0 : 0.5;
}

static void dispersion3(const model_t *m, const oracle_param *p, int nat, const double *xyz,
                        const double *trans, int ntr, double cutoff, double width,
                        const double *c6, const double *dc6dcn, double *energy,
                        double *dEdcn, double *gradient, double *sigma, int part, int nparts)
{
    /* get_atm_dispersion, atm.f90:433-825, called with rs9 = 4/3 and
     * alp + 2 (rational.f90:563, zero.f90:602) */
    double s9 = p->s9;
    if (fabs(s9) < EPS) return;
    double alp = p->alp + 2.0;
    double cutoff2 = cutoff * cutoff;
    double alp3 = alp / 3.0;
    int grad = dEdcn != NULL;
    int nid = m->nid;
#pragma omp parallel
    {
        double *el = calloc(nat, sizeof(double));
        double *dl = grad ? calloc(nat, sizeof(double)) : NULL;
        double *gl = grad ? calloc(3 * (size_t)nat, sizeof(double)) : NULL;
        double sl[9] = {0};
#pragma omp for schedule(dynamic, 1)
        for (int i = 0; i < nat; i++) {
            int izp = m->id[i];
            for (int j = 0; j <= i; j++) {
                if (!owns_pair(part, nparts, i, j)) continue;
                int jzp = m->id[j];
                double c6ij = c6[(size_t)j * nat + i];
                double r0ij = RS9 * m->rvdw[jzp * nid + izp];
                for (int jt = 0; jt < ntr; jt++) {
                    double vij[3];
                    for (int c = 0; c < 3; c++)
                        vij[c] = xyz[3 * j + c] + trans[3 * jt + c] - xyz[3 * i + c];
                    double r2ij = vij[0] * vij[0] + vij[1] * vij[1] + vij[2] * vij[2];
                    if (r2ij > cutoff2 || r2ij < EPS) continue;
                    double rij = sqrt(r2ij);
                    double swij, dswijdr;
                    smooth_cutoff(rij, cutoff, width, &swij, &dswijdr);
                    for (int k = 0; k <= j; k++) {
                        int kzp = m->id[k];
                        double c6ik = c6[(size_t)k * nat + i];
                        double c6jk = c6[(size_t)k * nat + j];
                        if (grad && (fabs(c6ij) < EPS || fabs(c6ik) < EPS || fabs(c6jk) < EPS))
                            continue;
                        double c9 = -s9 * sqrt(fabs(c6ij * c6ik * c6jk));
                        double r0ik = RS9 * m->rvdw[kzp * nid + izp];
                        double r0jk = RS9 * m->rvdw[kzp * nid + jzp];
                        double r0 = r0ij * r0ik * r0jk;
                        double triple = triple_scale(i, j, k);
                        for (int kt = 0; kt < ntr; kt++) {
                            double vik[3], vjk[3];
                            for (int c = 0; c < 3; c++)
                                vik[c] = xyz[3 * k + c] + trans[3 * kt + c] - xyz[3 * i + c];
                            double r2ik = vik[0] * vik[0] + vik[1] * vik[1] + vik[2] * vik[2];
                            if (r2ik > cutoff2 || r2ik < EPS) continue;
                            double rik = sqrt(r2ik);
                            double swik, dswikdr;
                            smooth_cutoff(rik, cutoff, width, &swik, &dswikdr);
                            for (int c = 0; c < 3; c++) vjk[c] = vik[c] - vij[c];
                            double r2jk = vjk[0] * vjk[0] + vjk[1] * vjk[1] + vjk[2] * vjk[2];
                            if (r2jk > cutoff2 || r2jk < EPS) continue;
                            double rjk = sqrt(r2jk);
                            double swjk, dswjkdr;
                            smooth_cutoff(rjk, cutoff, width, &swjk, &dswjkdr);
                            double sw = swij * swik * swjk;
                            double r2 = r2ij * r2ik * r2jk;
                            double r1 = sqrt(r2);
                            double r3 = r2 * r1;
                            double r5 = r3 * r2;
                            double fdmp = 1.0 / (1.0 + 6.0 * pow(r0 / r1, alp3));
                            double ang = 0.375 * (r2ij + r2jk - r2ik) * (r2ij - r2jk + r2ik)
                                       * (-r2ij + r2jk + r2ik) / r5 + 1.0 / r3;
                            double rr = ang * fdmp;
                            if (!grad) {
                                double dE = rr * c9 * triple * sw / 3.0;
                                el[i] -= dE; el[j] -= dE; el[k] -= dE;
                                continue;
                            }
                            double r0r1alp3 = pow(r0 / r1, alp3);
                            double dfdmp = -2.0 * alp * r0r1alp3 * (fdmp * fdmp);
                            double dang, dGij[3], dGik[3], dGjk[3];
                            dang = -0.375 * (r2ij * r2ij * r2ij + r2ij * r2ij * (r2jk + r2ik)
                                   + r2ij * (3.0 * r2jk * r2jk + 2.0 * r2jk * r2ik + 3.0 * r2ik * r2ik)
                                   - 5.0 * (r2jk - r2ik) * (r2jk - r2ik) * (r2jk + r2ik)) / r5;
                            double dE0 = rr * c9;
                            for (int c = 0; c < 3; c++)
                                dGij[c] = sw * c9 * (-dang * fdmp + ang * dfdmp) / r2ij * vij[c]
                                        - dE0 * dswijdr / rij * swik * swjk * vij[c];
                            dang = -0.375 * (r2ik * r2ik * r2ik + r2ik * r2ik * (r2jk + r2ij)
                                   + r2ik * (3.0 * r2jk * r2jk + 2.0 * r2jk * r2ij + 3.0 * r2ij * r2ij)
                                   - 5.0 * (r2jk - r2ij) * (r2jk - r2ij) * (r2jk + r2ij)) / r5;
                            for (int c = 0; c < 3; c++)
                                dGik[c] = sw * c9 * (-dang * fdmp + ang * dfdmp) / r2ik * vik[c]
                                        - dE0 * dswikdr / rik * swij * swjk * vik[c];
                            dang = -0.375 * (r2jk * r2jk * r2jk + r2jk * r2jk * (r2ik + r2ij)
                                   + r2jk * (3.0 * r2ik * r2ik + 2.0 * r2ik * r2ij + 3.0 * r2ij * r2ij)
                                   - 5.0 * (r2ik - r2ij) * (r2ik - r2ij) * (r2ik + r2ij)) / r5;
                            for (int c = 0; c < 3; c++)
                                dGjk[c] = sw * c9 * (-dang * fdmp + ang * dfdmp) / r2jk * vjk[c]
                                        - dE0 * dswjkdr / rjk * swij * swik * vjk[c];
                            double dE = dE0 * triple * sw;
                            el[i] -= dE / 3.0; el[j] -= dE / 3.0; el[k] -= dE / 3.0;
                            for (int c = 0; c < 3; c++) {
                                gl[3 * i + c] -= (dGij[c] + dGik[c]) * triple;
                                gl[3 * j + c] += (dGij[c] - dGjk[c]) * triple;
                                gl[3 * k + c] += (dGik[c] + dGjk[c]) * triple;
                            }
                            for (int a = 0; a < 3; a++)
                                for (int b = 0; b < 3; b++)
                                    sl[a + 3 * b] += (dGij[a] * vij[b] + dGik[a] * vik[b]
                                                      + dGjk[a] * vjk[b]) * triple;
                            dl[i] -= dE * 0.5 * (dc6dcn[(size_t)i * nat + j] / c6ij
                                                 + dc6dcn[(size_t)i * nat + k] / c6ik);
                            dl[j] -= dE * 0.5 * (dc6dcn[(size_t)j * nat + i] / c6ij
                                                 + dc6dcn[(size_t)j * nat + k] / c6jk);
                            dl[k] -= dE * 0.5 * (dc6dcn[(size_t)k * nat + i] / c6ik
                                                 + dc6dcn[(size_t)k * nat + j] / c6jk);
                        }
                    }
                }
            }
        }
#pragma omp critical(oracle_disp3)
        {
            for (int i = 0; i < nat; i++) energy[i] += el[i];
            if (grad) {
                for (int i = 0; i < nat; i++) dEdcn[i] += dl[i];
                for (int k = 0; k < 3 * nat; k++) gradient[k] += gl[k];
                for (int k = 0; k < 9; k++) sigma[k] += sl[k];
            }
        }
        free(el); free(dl); free(gl);
    }
}

/* ------------------------------------------------------------- pipeline -- */

/* ------------------------------------------------------------- pairwise -- */

static void pairwise2(const model_t *m, const oracle_param *p, int nat, const double *xyz,
                      const double *trans, int ntr, double cutoff, double width, const double *c6,
                      double *energy)
{
    /* get_pairwise_dispersion2 of each family: rational.f90:623-705,
     * zero.f90:662-755, mzero.f90, optimizedpower.f90, cso.f90, z.f90 (the
     * energy expressions of the dispersion loops, without derivatives);
     * energy[i][j] gets half of every (i, j, T) pair energy, energy[j][i] the
     * other half, a self pair (j = i, T != 0) its half once */
    double cutoff2 = cutoff * cutoff;
    double alp6 = p->alp, alp8 = p->alp + 2.0;
    for (int i = 0; i < nat; i++) {
        int izp = m->id[i];
        for (int j = 0; j <= i; j++) {
            int jzp = m->id[j];
            double rrij = 3 * m->r4r2[izp] * m->r4r2[jzp];
            double c6ij = c6[(size_t)j * nat + i];
            double rvdw = m->rvdw[jzp * m->nid + izp];
            for (int t = 0; t < ntr; t++) {
                double v[3];
                for (int c = 0; c < 3; c++) v[c] = xyz[3 * i + c] - (xyz[3 * j + c] + trans[3 * t + c]);
                double r2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
                if (r2 > cutoff2 || r2 < EPS) continue;
                double r1 = sqrt(r2);
                double sw, dswdr;
                smooth_cutoff(r1, cutoff, width, &sw, &dswdr);
                double r4 = r2 * r2, r6 = r4 * r2, r8 = r6 * r2, e0;
                switch (p->damping) {
                case ORACLE_RATIONAL: {
                    double r0 = p->a1 * sqrt(rrij) + p->a2;
                    double t6 = 1.0 / (r6 + pow(r0, 6)), t8 = 1.0 / (r8 + pow(r0, 8));
                    e0 = p->s6 * t6 + p->s8 * rrij * t8;
                    break;
                }
                case ORACLE_ZERO: {
                    double t6 = pow(p->rs6 * rvdw / r1, alp6), t8 = pow(p->rs8 * rvdw / r1, alp8);
                    e0 = p->s6 / (1.0 + 6.0 * t6) / r6 + p->s8 * rrij / (1.0 + 6.0 * t8) / r8;
                    break;
                }
                case ORACLE_MZERO: {
                    double t6 = pow(r1 / (p->rs6 * rvdw) + p->bet * rvdw, -alp6);
                    double t8 = pow(r1 / (p->rs8 * rvdw) + p->bet * rvdw, -alp8);
                    e0 = p->s6 / (1.0 + 6.0 * t6) / r6 + p->s8 * rrij / (1.0 + 6.0 * t8) / r8;
                    break;
                }
                case ORACLE_OPTIMIZEDPOWER: {
                    double r0 = p->a1 * sqrt(rrij) + p->a2, ab = pow(r0, p->bet), rb = pow(r2, p->bet * 0.5);
                    double t6 = rb / (rb * r6 + ab * pow(r0, 6)), t8 = rb / (rb * r8 + ab * pow(r0, 8));
                    e0 = p->s6 * t6 + p->s8 * rrij * t8;
                    break;
                }
                case ORACLE_CSO: {
                    double r0 = sqrt(rrij);
                    double sf = 1.0 / (1.0 + exp(r1 - p->a2 * r0));
                    e0 = (p->s6 + p->a1 * sf) / (r6 + pow(p->rs6 * r0 + p->rs8, 6));
                    break;
                }
                default: {
                    double zc = p->a1 / (double)((izp + 1) + (jzp + 1)) * c6ij;
                    e0 = p->s6 / (r6 + zc) + p->s8 * rrij / (r8 + zc * rrij);
                    break;
                }
                }
                double dE = -c6ij * sw * e0 * 0.5;
                energy[(size_t)i * nat + j] += dE;
                if (i != j) energy[(size_t)j * nat + i] += dE;
            }
        }
    }
}

static void pairwise3(const model_t *m, const oracle_param *p, int nat, const double *xyz,
                      const double *trans, int ntr, double cutoff, double width, const double *c6,
                      double *energy)
{
    /* get_atm_pairwise_dispersion, atm.f90:829-950 with rs9 = 4/3 and alp + 2:
     * a sixth of every triple energy to each ordered pair of the triple */
    if (fabs(p->s9) < EPS) return;
    double cutoff2 = cutoff * cutoff;
    double alp3 = (p->alp + 2.0) / 3.0;
    for (int i = 0; i < nat; i++) {
        int izp = m->id[i];
        for (int j = 0; j <= i; j++) {
            int jzp = m->id[j];
            double c6ij = c6[(size_t)j * nat + i];
            double r0ij = RS9 * m->rvdw[jzp * m->nid + izp];
            for (int jt = 0; jt < ntr; jt++) {
                double vij[3];
                for (int c = 0; c < 3; c++) vij[c] = xyz[3 * j + c] + trans[3 * jt + c] - xyz[3 * i + c];
                double r2ij = vij[0] * vij[0] + vij[1] * vij[1] + vij[2] * vij[2];
                if (r2ij > cutoff2 || r2ij < EPS) continue;
                double rij = sqrt(r2ij), swij, dsw;
                smooth_cutoff(rij, cutoff, width, &swij, &dsw);
                for (int k = 0; k <= j; k++) {
                    int kzp = m->id[k];
                    double c6ik = c6[(size_t)k * nat + i], c6jk = c6[(size_t)k * nat + j];
                    double c9 = -p->s9 * sqrt(fabs(c6ij * c6ik * c6jk));
                    double r0 = r0ij * RS9 * m->rvdw[kzp * m->nid + izp] * RS9 * m->rvdw[kzp * m->nid + jzp];
                    double triple = triple_scale(i, j, k);
                    for (int kt = 0; kt < ntr; kt++) {
                        double vik[3], vjk[3];
                        for (int c = 0; c < 3; c++) vik[c] = xyz[3 * k + c] + trans[3 * kt + c] - xyz[3 * i + c];
                        double r2ik = vik[0] * vik[0] + vik[1] * vik[1] + vik[2] * vik[2];
                        if (r2ik > cutoff2 || r2ik < EPS) continue;
                        double rik = sqrt(r2ik), swik;
                        smooth_cutoff(rik, cutoff, width, &swik, &dsw);
                        for (int c = 0; c < 3; c++) vjk[c] = vik[c] - vij[c];
                        double r2jk = vjk[0] * vjk[0] + vjk[1] * vjk[1] + vjk[2] * vjk[2];
                        if (r2jk > cutoff2 || r2jk < EPS) continue;
                        double rjk = sqrt(r2jk), swjk;
                        smooth_cutoff(rjk, cutoff, width, &swjk, &dsw);
                        double sw = swij * swik * swjk;
                        double r2 = r2ij * r2ik * r2jk, r1 = sqrt(r2), r3 = r2 * r1, r5 = r3 * r2;
                        double fdmp = 1.0 / (1.0 + 6.0 * pow(r0 / r1, alp3));
                        double ang = 0.375 * (r2ij + r2jk - r2ik) * (r2ij - r2jk + r2ik) * (-r2ij + r2jk + r2ik) / r5
                                   + 1.0 / r3;
                        double dE = ang * fdmp * c9 * triple * sw / 6.0;
                        energy[(size_t)i * nat + j] -= dE; energy[(size_t)i * nat + k] -= dE;
                        energy[(size_t)j * nat + i] -= dE; energy[(size_t)j * nat + k] -= dE;
                        energy[(size_t)k * nat + i] -= dE; energy[(size_t)k * nat + j] -= dE;
                    }
                }
            }
        }
    }
}

int oracle_get_pairwise_dispersion(int nat, const int *numbers, const double *xyz, const double *lattice,
                                   const int *periodic, const int *ghost, const oracle_param *param,
                                   const oracle_cutoff *cutoff, double *pair2, double *pair3)
{
    /* get_pairwise_dispersion_v2, disp.f90:403-457 */
    if (param->damping < ORACLE_RATIONAL || param->damping > ORACLE_Z) return 4;
    model_t m;
    if (model_new(&m, nat, numbers, ghost)) return 1;
    double zero[9] = {0};
    int per0[3] = {0, 0, 0};
    const double *lat = lattice ? lattice : zero;
    const int *per = periodic ? periodic : per0;
    int ntr;
    double *cn = malloc(sizeof(double) * (nat > 0 ? nat : 1));
    double *trans = lattice_points(lat, per, cutoff->cn, &ntr);
    partitioned_cn(nat, xyz, m.id, m.rcov, trans, ntr, cutoff->cn, cn, 0, 1);
    free(trans);
    double *gwvec = malloc(sizeof(double) * (size_t)(nat > 0 ? nat : 1) * m.mref);
    weight_references(&m, nat, cn, gwvec, NULL);
    size_t nn = (size_t)nat * nat;
    double *c6 = malloc(sizeof(double) * (nn > 0 ? nn : 1));
    get_atomic_c6(&m, nat, gwvec, NULL, c6, NULL, 0, 1);
    memset(pair2, 0, sizeof(double) * nn);
    memset(pair3, 0, sizeof(double) * nn);
    trans = lattice_points(lat, per, cutoff->disp2, &ntr);
    pairwise2(&m, param, nat, xyz, trans, ntr, cutoff->disp2, cutoff->width2, c6, pair2);
    free(trans);
    trans = lattice_points(lat, per, cutoff->disp3, &ntr);
    pairwise3(&m, param, nat, xyz, trans, ntr, cutoff->disp3, cutoff->width3, c6, pair3);
    free(trans);
    free(cn); free(gwvec); free(c6);
    model_free(&m);
    return 0;
}

/* -------------------------------------------------------------- hessian -- */

static void weight_references2(const model_t *m, int nat, const double *cn, double *gwvec,
                               double *gwdcn, double *gwd2cn)
{
    /* model.f90:201-273, the branch with second derivatives */
    int mref = m->mref;
    double wf2 = 2 * WF;
    for (int k = 0; k < nat * mref; k++) gwvec[k] = gwdcn[k] = gwd2cn[k] = 0.0;
    for (int i = 0; i < nat; i++) {
        int izp = m->id[i];
        int nref = m->ref[izp];
        const double *cnref = m->cn + izp * mref;
        double gwt[D3_MAX_REF];
        double norm = 0.0, dnorm = 0.0, d2norm = 0.0;
        for (int r = 0; r < nref; r++) {
            double gw = exp(-WF * (cn[i] - cnref[r]) * (cn[i] - cnref[r]));
            gwt[r] = gw;
            double dcn = cnref[r] - cn[i];
            norm += gw;
            dnorm += wf2 * dcn * gw;
            d2norm += (wf2 * wf2 * dcn * dcn - wf2) * gw;
        }
        norm = 1.0 / norm;
        double maxcn = cnref[0];
        for (int r = 1; r < nref; r++) if (cnref[r] > maxcn) maxcn = cnref[r];
        for (int r = 0; r < nref; r++) {
            double expw = gwt[r];
            double dcn = cnref[r] - cn[i];
            double expd = wf2 * dcn * expw;
            double expdd = (wf2 * wf2 * dcn * dcn - wf2) * expw;
            double gwk = expw * norm;
            if (is_exceptional(gwk)) gwk = (maxcn == cnref[r]) ? 1.0 : 0.0;
            gwvec[i * mref + r] = gwk;
            double dgwk = expd * norm - expw * dnorm * (norm * norm);
            if (is_exceptional(dgwk)) dgwk = 0.0;
            gwdcn[i * mref + r] = dgwk;
            double d2gwk = expdd * norm - 2.0 * expd * dnorm * (norm * norm) - expw * d2norm * (norm * norm)
                         + 2.0 * expw * dnorm * dnorm * (norm * norm * norm);
            if (is_exceptional(d2gwk)) d2gwk = 0.0;
            gwd2cn[i * mref + r] = d2gwk;
        }
    }
}

static void get_atomic_c6_2(const model_t *m, int nat, const double *gw, const double *dgw, const double *d2gw,
                            double *c6, double *dc6dcn, double *d2c6dcn2, double *d2c6dcnij)
{
    /* model.f90:363-401: C6, dC6/dCN and the second derivatives; element
     * (iat, jat) of each matrix at [iat*nat + jat] */
    int mref = m->mref, nid = m->nid;
    size_t nn = (size_t)nat * nat;
    memset(c6, 0, sizeof(double) * nn);
    memset(dc6dcn, 0, sizeof(double) * nn);
    memset(d2c6dcn2, 0, sizeof(double) * nn);
    memset(d2c6dcnij, 0, sizeof(double) * nn);
    for (int i = 0; i < nat; i++) {
        if (m->ghost[i]) continue;
        int izp = m->id[i];
        for (int j = 0; j <= i; j++) {
            if (m->ghost[j]) continue;
            int jzp = m->id[j];
            double v = 0, di = 0, dj = 0, d2i = 0, d2j = 0, dmix = 0;
            for (int ir = 0; ir < m->ref[izp]; ir++)
                for (int jr = 0; jr < m->ref[jzp]; jr++) {
                    double refc6 = m->c6[(((size_t)izp * nid + jzp) * mref + ir) * mref + jr];
                    v += gw[i * mref + ir] * gw[j * mref + jr] * refc6;
                    di += dgw[i * mref + ir] * gw[j * mref + jr] * refc6;
                    dj += gw[i * mref + ir] * dgw[j * mref + jr] * refc6;
                    d2i += d2gw[i * mref + ir] * gw[j * mref + jr] * refc6;
                    d2j += gw[i * mref + ir] * d2gw[j * mref + jr] * refc6;
                    dmix += dgw[i * mref + ir] * dgw[j * mref + jr] * refc6;
                }
            c6[(size_t)i * nat + j] = c6[(size_t)j * nat + i] = v;
            dc6dcn[(size_t)i * nat + j] = di;
            dc6dcn[(size_t)j * nat + i] = dj;
            d2c6dcn2[(size_t)i * nat + j] = d2i;
            d2c6dcn2[(size_t)j * nat + i] = d2j;
            d2c6dcnij[(size_t)i * nat + j] = d2c6dcnij[(size_t)j * nat + i] = dmix;
        }
    }
}

static void cn_with_derivs(int nat, const double *xyz, const int *id, const double *rcov, const double *trans,
                           int ntr, double cutoff, double *cn, double *dr)
{
    /* the coordination number (ncoord.f90:86-144) and dr[(3a+c)*nat + k] =
     * dCN_k/dR_a,c, the derivative the reference takes from mctc-lib's
     * counting-function CN (ncoord.f90:30-58) */
    double cutoff2 = cutoff * cutoff;
    memset(cn, 0, sizeof(double) * nat);
    memset(dr, 0, sizeof(double) * 3 * (size_t)nat * nat);
    for (int i = 0; i < nat; i++) {
        int izp = id[i];
        for (int j = 0; j <= i; j++) {
            int jzp = id[j];
            double rc = rcov[izp] + rcov[jzp];
            for (int t = 0; t < ntr; t++) {
                double v[3];
                for (int c = 0; c < 3; c++) v[c] = xyz[3 * i + c] - (xyz[3 * j + c] + trans[3 * t + c]);
                double r2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
                if (r2 > cutoff2 || r2 < 1.0e-12) continue;
                double r1 = sqrt(r2);
                double cf = 1.0 / (1.0 + exp(-KCN * (rc / r1 - 1.0)));
                cn[i] += cf;
                if (i == j) continue;
                cn[j] += cf;
                double dcf = -cf * (1.0 - cf) * KCN * rc / r2;
                for (int c = 0; c < 3; c++) {
                    double dg = dcf * v[c] / r1;
                    dr[(size_t)(3 * i + c) * nat + i] += dg;
                    dr[(size_t)(3 * i + c) * nat + j] += dg;
                    dr[(size_t)(3 * j + c) * nat + i] -= dg;
                    dr[(size_t)(3 * j + c) * nat + j] -= dg;
                }
            }
        }
    }
}

static void smooth_cutoff_r2(double r2, double cutoff, double width, double *sw, double *dsw, double *d2sw)
{
    /* cutoff.f90:104-134: the switch and its first two derivatives with
     * respect to the squared distance */
    double r1 = sqrt(r2), dswdr = 0.0, d2swdr2 = 0.0;
    if (width <= 0.0 || width >= cutoff) {
        *sw = 1.0;
    } else {
        double inner = cutoff - width;
        if (r1 <= inner) {
            *sw = 1.0;
        } else if (r1 >= cutoff) {
            *sw = 0.0;
        } else {
            double x = (cutoff - r1) / width;
            *sw = x * x * x * (10.0 + x * (-15.0 + 6.0 * x));
            dswdr = -30.0 * x * x * (1.0 - x) * (1.0 - x) / width;
            d2swdr2 = 60.0 * x * (1.0 - x) * (1.0 - 2.0 * x) / (width * width);
        }
    }
    *dsw = 0.5 * dswdr / r1;
    *d2sw = 0.25 * (d2swdr2 - dswdr / r1) / r2;
}

static void damping_kernel(const model_t *m, const oracle_param *p, int izp, int jzp, double r2, double c6,
                           double k[6])
{
    /* get_damping_kernel of each family (rational.f90, zero.f90, mzero.f90,
     * optimizedpower.f90, cso.f90, z.f90): the pair energy e = -C6 p(u) with
     * u = r^2 and its derivatives e_u, e_c, e_uu, e_uc, e_cc */
    for (int q = 0; q < 6; q++) k[q] = 0.0;
    if (p->damping != ORACLE_CSO && fabs(p->s6) < EPS && fabs(p->s8) < EPS) return;
    double u = r2;
    double rrij = 3 * m->r4r2[izp] * m->r4r2[jzp];
    double rvdw = m->rvdw[jzp * m->nid + izp];
    double pv, pd, pdd, pc = 0.0, puc = 0.0, pcc = 0.0;
    switch (p->damping) {
    case ORACLE_RATIONAL: {
        double r0 = p->a1 * sqrt(rrij) + p->a2, r02 = r0 * r0, r06 = r02 * r02 * r02, r08 = r06 * r02;
        double t6 = 1.0 / (u * u * u + r06), t8 = 1.0 / (u * u * u * u + r08);
        double t6d = -3.0 * u * u * t6 * t6, t8d = -4.0 * u * u * u * t8 * t8;
        double t6dd = -6.0 * u * t6 * t6 + 18.0 * pow(u, 4) * pow(t6, 3);
        double t8dd = -12.0 * u * u * t8 * t8 + 32.0 * pow(u, 6) * pow(t8, 3);
        pv = p->s6 * t6 + p->s8 * rrij * t8;
        pd = p->s6 * t6d + p->s8 * rrij * t8d;
        pdd = p->s6 * t6dd + p->s8 * rrij * t8dd;
        break;
    }
    case ORACLE_ZERO:
    case ORACLE_MZERO: {
        double alp6 = p->alp, alp8 = p->alp + 2.0;
        double t6, t8, t6d, t8d, t6dd, t8dd;
        if (p->damping == ORACLE_ZERO) {
            double a6 = 0.5 * alp6, a8 = 0.5 * alp8;
            t6 = pow(p->rs6 * rvdw / sqrt(u), alp6);
            t8 = pow(p->rs8 * rvdw / sqrt(u), alp8);
            t6d = -a6 * t6 / u;
            t8d = -a8 * t8 / u;
            t6dd = a6 * (a6 + 1.0) * t6 / (u * u);
            t8dd = a8 * (a8 + 1.0) * t8 / (u * u);
        } else {
            double r1 = sqrt(u), betr0 = p->bet * rvdw;
            double w6 = r1 / (p->rs6 * rvdw) + betr0, w8 = r1 / (p->rs8 * rvdw) + betr0;
            double w6d = 1.0 / (p->rs6 * rvdw * 2.0 * r1), w8d = 1.0 / (p->rs8 * rvdw * 2.0 * r1);
            double w6dd = -1.0 / (p->rs6 * rvdw * 4.0 * u * r1), w8dd = -1.0 / (p->rs8 * rvdw * 4.0 * u * r1);
            t6 = pow(w6, -alp6);
            t8 = pow(w8, -alp8);
            t6d = -alp6 * pow(w6, -alp6 - 1.0) * w6d;
            t8d = -alp8 * pow(w8, -alp8 - 1.0) * w8d;
            t6dd = alp6 * (alp6 + 1.0) * pow(w6, -alp6 - 2.0) * w6d * w6d - alp6 * pow(w6, -alp6 - 1.0) * w6dd;
            t8dd = alp8 * (alp8 + 1.0) * pow(w8, -alp8 - 2.0) * w8d * w8d - alp8 * pow(w8, -alp8 - 1.0) * w8dd;
        }
        double f6 = 1.0 / (1.0 + 6.0 * t6), f8 = 1.0 / (1.0 + 6.0 * t8);
        double f6d = -6.0 * t6d * f6 * f6, f8d = -6.0 * t8d * f8 * f8;
        double f6dd = -6.0 * t6dd * f6 * f6 + 72.0 * t6d * t6d * pow(f6, 3);
        double f8dd = -6.0 * t8dd * f8 * f8 + 72.0 * t8d * t8d * pow(f8, 3);
        double c6t = f6 / pow(u, 3), c6td = f6d / pow(u, 3) - 3.0 * f6 / pow(u, 4);
        double c6tdd = f6dd / pow(u, 3) - 6.0 * f6d / pow(u, 4) + 12.0 * f6 / pow(u, 5);
        double c8t = f8 / pow(u, 4), c8td = f8d / pow(u, 4) - 4.0 * f8 / pow(u, 5);
        double c8tdd = f8dd / pow(u, 4) - 8.0 * f8d / pow(u, 5) + 20.0 * f8 / pow(u, 6);
        pv = p->s6 * c6t + p->s8 * rrij * c8t;
        pd = p->s6 * c6td + p->s8 * rrij * c8td;
        pdd = p->s6 * c6tdd + p->s8 * rrij * c8tdd;
        break;
    }
    case ORACLE_OPTIMIZEDPOWER: {
        double r0 = p->a1 * sqrt(rrij) + p->a2, r02 = r0 * r0, r06 = r02 * r02 * r02, r08 = r06 * r02;
        double ab = pow(r0, p->bet), a6 = ab * r06, a8 = ab * r08, q = 0.5 * p->bet;
        double d6 = pow(u, 3) + a6 * pow(u, -q), d8 = pow(u, 4) + a8 * pow(u, -q);
        double d6d = 3.0 * u * u - q * a6 * pow(u, -q - 1.0), d8d = 4.0 * pow(u, 3) - q * a8 * pow(u, -q - 1.0);
        double d6dd = 6.0 * u + q * (q + 1.0) * a6 * pow(u, -q - 2.0);
        double d8dd = 12.0 * u * u + q * (q + 1.0) * a8 * pow(u, -q - 2.0);
        double t6 = 1.0 / d6, t8 = 1.0 / d8;
        double t6d = -d6d * t6 * t6, t8d = -d8d * t8 * t8;
        double t6dd = -d6dd * t6 * t6 + 2.0 * d6d * d6d * pow(t6, 3);
        double t8dd = -d8dd * t8 * t8 + 2.0 * d8d * d8d * pow(t8, 3);
        pv = p->s6 * t6 + p->s8 * rrij * t8;
        pd = p->s6 * t6d + p->s8 * rrij * t8d;
        pdd = p->s6 * t6dd + p->s8 * rrij * t8dd;
        break;
    }
    case ORACLE_CSO: {
        double r1 = sqrt(u), r0 = sqrt(rrij);
        double dd6_6 = pow(p->rs6 * r0 + p->rs8, 6);
        double ef = exp(r1 - p->a2 * r0), sf = 1.0 / (1.0 + ef);
        double sfd = -sf * (1.0 - sf), sfdd = sf * (1.0 - sf) * (1.0 - 2.0 * sf);
        double sig = p->s6 + p->a1 * sf, sigd = p->a1 * sfd, sigdd = p->a1 * sfdd;
        double sigu = 0.5 * sigd / r1, siguu = 0.25 * sigdd / u - 0.25 * sigd / (u * r1);
        double t6 = 1.0 / (u * u * u + dd6_6);
        double t6d = -3.0 * u * u * t6 * t6, t6dd = -6.0 * u * t6 * t6 + 18.0 * pow(u, 4) * pow(t6, 3);
        pv = sig * t6;
        pd = sigu * t6 + sig * t6d;
        pdd = siguu * t6 + 2.0 * sigu * t6d + sig * t6dd;
        break;
    }
    default: {
        double r0 = p->a1 / (double)((izp + 1) + (jzp + 1)), b8 = r0 * rrij;
        double t6 = 1.0 / (u * u * u + r0 * c6), t8 = 1.0 / (u * u * u * u + b8 * c6);
        double t6u = -3.0 * u * u * t6 * t6, t8u = -4.0 * pow(u, 3) * t8 * t8;
        double t6uu = -6.0 * u * t6 * t6 + 18.0 * pow(u, 4) * pow(t6, 3);
        double t8uu = -12.0 * u * u * t8 * t8 + 32.0 * pow(u, 6) * pow(t8, 3);
        double t6c = -r0 * t6 * t6, t8c = -b8 * t8 * t8;
        double t6uc = 6.0 * u * u * r0 * pow(t6, 3), t8uc = 8.0 * pow(u, 3) * b8 * pow(t8, 3);
        double t6cc = 2.0 * r0 * r0 * pow(t6, 3), t8cc = 2.0 * b8 * b8 * pow(t8, 3);
        pv = p->s6 * t6 + p->s8 * rrij * t8;
        pd = p->s6 * t6u + p->s8 * rrij * t8u;
        pdd = p->s6 * t6uu + p->s8 * rrij * t8uu;
        pc = p->s6 * t6c + p->s8 * rrij * t8c;
        puc = p->s6 * t6uc + p->s8 * rrij * t8uc;
        pcc = p->s6 * t6cc + p->s8 * rrij * t8cc;
        break;
    }
    }
    k[0] = -c6 * pv;
    k[1] = -c6 * pd;
    k[2] = -pv - c6 * pc;
    k[3] = -c6 * pdd;
    k[4] = -pd - c6 * puc;
    k[5] = -2.0 * pc - c6 * pcc;
}

static void hessian2(const model_t *m, const oracle_param *p, int nat, const double *xyz, const double *trans,
                     int ntr, double cutoff, double width, const double *c6, const double *dc6dcn,
                     const double *d2c6dcn2, const double *d2c6dcnij, double *H, double *dEdcn, double *A,
                     double *D, int part, int nparts)
{
    /* get_dispersion2_hessian, damping.f90:393-539: the geometric blocks
     * into H [3N][3N], dE/dCN, d2E/dR dCN into A [3N][N] and d2E/dCN2 into
     * D [N][N] */
    size_t n3 = 3 * (size_t)nat;
    double cutoff2 = cutoff * cutoff;
    for (int i = 0; i < nat; i++) {
        int izp = m->id[i];
        for (int j = 0; j <= i; j++) {
            if (!owns_pair(part, nparts, i, j)) continue;
            int jzp = m->id[j];
            double c6ij = c6[(size_t)j * nat + i];
            double fac;
            int nc, cnat[2];
            double cnd[2], cnd2[2][2];
            if (i != j) {
                fac = 1.0; nc = 2; cnat[0] = i; cnat[1] = j;
                cnd[0] = dc6dcn[(size_t)i * nat + j];
                cnd[1] = dc6dcn[(size_t)j * nat + i];
                cnd2[0][0] = d2c6dcn2[(size_t)i * nat + j];
                cnd2[1][1] = d2c6dcn2[(size_t)j * nat + i];
                cnd2[0][1] = cnd2[1][0] = d2c6dcnij[(size_t)i * nat + j];
            } else {
                fac = 0.5; nc = 1; cnat[0] = i;
                cnd[0] = 2.0 * dc6dcn[(size_t)i * nat + i];
                cnd2[0][0] = 2.0 * d2c6dcn2[(size_t)i * nat + i] + 2.0 * d2c6dcnij[(size_t)i * nat + i];
            }
            for (int t = 0; t < ntr; t++) {
                double v[3];
                for (int c = 0; c < 3; c++) v[c] = xyz[3 * i + c] - (xyz[3 * j + c] + trans[3 * t + c]);
                double r2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
                if (r2 > cutoff2 || r2 < EPS) continue;
                double k[6], sw, swr, swrr;
                damping_kernel(m, p, izp, jzp, r2, c6ij, k);
                smooth_cutoff_r2(r2, cutoff, width, &sw, &swr, &swrr);
                double fr = fac * (swr * k[0] + sw * k[1]);
                double frr = fac * (swrr * k[0] + 2.0 * swr * k[1] + sw * k[3]);
                double fc = fac * sw * k[2];
                double frc = fac * (swr * k[2] + sw * k[4]);
                double fcc = fac * sw * k[5];
                if (i != j) {
                    for (int a = 0; a < 3; a++)
                        for (int b = 0; b < 3; b++) {
                            double blk = 4.0 * frr * v[a] * v[b] + (a == b ? 2.0 * fr : 0.0);
                            H[(3 * i + a) * n3 + 3 * i + b] += blk;
                            H[(3 * j + a) * n3 + 3 * j + b] += blk;
                            H[(3 * i + a) * n3 + 3 * j + b] -= blk;
                            H[(3 * j + a) * n3 + 3 * i + b] -= blk;
                        }
                }
                for (int ia = 0; ia < nc; ia++) {
                    dEdcn[cnat[ia]] += fc * cnd[ia];
                    for (int ib = 0; ib < nc; ib++)
                        D[(size_t)cnat[ia] * nat + cnat[ib]] += fcc * cnd[ia] * cnd[ib] + fc * cnd2[ia][ib];
                }
                if (i != j) {
                    for (int ia = 0; ia < nc; ia++)
                        for (int c = 0; c < 3; c++) {
                            A[(size_t)(3 * i + c) * nat + cnat[ia]] += frc * 2.0 * v[c] * cnd[ia];
                            A[(size_t)(3 * j + c) * nat + cnat[ia]] -= frc * 2.0 * v[c] * cnd[ia];
                        }
                }
            }
        }
    }
}

static void hessian3(const model_t *m, const oracle_param *p, int nat, const double *xyz, const double *trans,
                     int ntr, double cutoff, double width, const double *c6, const double *dc6dcn,
                     const double *d2c6dcn2, const double *d2c6dcnij, double *H, double *dEdcn, double *A,
                     double *D, int part, int nparts)
{
    /* get_atm_dispersion_hessian, atm.f90:38-429, with rs9 = 4/3 and alp + 2 */
    if (fabs(p->s9) < EPS) return;
    static const int sigp[3][3] = {{-1, -1, 0}, {1, 0, -1}, {0, 1, 1}};      /* [atom][pair] */
    static const double cl[3][3] = {{1, -1, 1}, {1, 1, -1}, {-1, 1, 1}};    /* [l][pair] */
    size_t n3 = 3 * (size_t)nat;
    double cutoff2 = cutoff * cutoff;
    double alp3 = (p->alp + 2.0) / 3.0, aexp = 0.5 * alp3;
    for (int i = 0; i < nat; i++) {
        int izp = m->id[i];
        for (int j = 0; j <= i; j++) {
            if (!owns_pair(part, nparts, i, j)) continue;
            int jzp = m->id[j];
            for (int jt = 0; jt < ntr; jt++) {
                double vec[3][3], u[3];
                for (int c = 0; c < 3; c++) vec[0][c] = xyz[3 * j + c] + trans[3 * jt + c] - xyz[3 * i + c];
                u[0] = vec[0][0] * vec[0][0] + vec[0][1] * vec[0][1] + vec[0][2] * vec[0][2];
                if (u[0] > cutoff2 || u[0] < EPS) continue;
                for (int kk = 0; kk <= j; kk++) {
                    int kzp = m->id[kk];
                    double triple = triple_scale(i, j, kk);
                    double r0 = RS9 * m->rvdw[jzp * m->nid + izp] * RS9 * m->rvdw[kzp * m->nid + izp]
                              * RS9 * m->rvdw[kzp * m->nid + jzp];
                    for (int kt = 0; kt < ntr; kt++) {
                        for (int c = 0; c < 3; c++) vec[1][c] = xyz[3 * kk + c] + trans[3 * kt + c] - xyz[3 * i + c];
                        u[1] = vec[1][0] * vec[1][0] + vec[1][1] * vec[1][1] + vec[1][2] * vec[1][2];
                        if (u[1] > cutoff2 || u[1] < EPS) continue;
                        for (int c = 0; c < 3; c++) vec[2][c] = vec[1][c] - vec[0][c];
                        u[2] = vec[2][0] * vec[2][0] + vec[2][1] * vec[2][1] + vec[2][2] * vec[2][2];
                        if (u[2] > cutoff2 || u[2] < EPS) continue;
                        double c6t[3] = {c6[(size_t)j * nat + i], c6[(size_t)kk * nat + i], c6[(size_t)kk * nat + j]};
                        if (fabs(c6t[0]) < EPS || fabs(c6t[1]) < EPS || fabs(c6t[2]) < EPS) continue;
                        double swp[3], dswp[3], d2swp[3];
                        for (int q = 0; q < 3; q++) smooth_cutoff_r2(u[q], cutoff, width, &swp[q], &dswp[q], &d2swp[q]);
                        double sval = swp[0] * swp[1] * swp[2];
                        double sp[3] = {dswp[0] * swp[1] * swp[2], swp[0] * dswp[1] * swp[2], swp[0] * swp[1] * dswp[2]};
                        double spq[3][3];
                        spq[0][0] = d2swp[0] * swp[1] * swp[2];
                        spq[1][1] = swp[0] * d2swp[1] * swp[2];
                        spq[2][2] = swp[0] * swp[1] * d2swp[2];
                        spq[0][1] = spq[1][0] = dswp[0] * dswp[1] * swp[2];
                        spq[0][2] = spq[2][0] = dswp[0] * swp[1] * dswp[2];
                        spq[1][2] = spq[2][1] = swp[0] * dswp[1] * dswp[2];
                        double ww = u[0] * u[1] * u[2];
                        double wp[3] = {u[1] * u[2], u[0] * u[2], u[0] * u[1]};
                        double wpq[3][3] = {{0, u[2], u[1]}, {u[2], 0, u[0]}, {u[1], u[0], 0}};
                        double lval[3] = {u[0] + u[2] - u[1], u[0] - u[2] + u[1], -u[0] + u[2] + u[1]};
                        double nval = lval[0] * lval[1] * lval[2];
                        double np[3], npq[3][3];
                        for (int a = 0; a < 3; a++)
                            np[a] = cl[0][a] * lval[1] * lval[2] + cl[1][a] * lval[0] * lval[2]
                                  + cl[2][a] * lval[0] * lval[1];
                        for (int a = 0; a < 3; a++)
                            for (int b = 0; b < 3; b++) {
                                double tmp = 0.0;
                                for (int il = 0; il < 3; il++)
                                    for (int im = 0; im < 3; im++) {
                                        if (il == im) continue;
                                        tmp += cl[il][a] * cl[im][b] * lval[3 - il - im];
                                    }
                                npq[a][b] = tmp;
                            }
                        double gv = pow(ww, -2.5), gd = -2.5 * pow(ww, -3.5), gdd = 8.75 * pow(ww, -4.5);
                        double hv = pow(ww, -1.5), hd = -1.5 * pow(ww, -2.5), hdd = 3.75 * pow(ww, -3.5);
                        double ang = 0.375 * nval * gv + hv, angp[3], angpq[3][3];
                        for (int a = 0; a < 3; a++) angp[a] = 0.375 * (np[a] * gv + nval * gd * wp[a]) + hd * wp[a];
                        for (int a = 0; a < 3; a++)
                            for (int b = 0; b < 3; b++)
                                angpq[a][b] = 0.375 * (npq[a][b] * gv + np[a] * gd * wp[b] + np[b] * gd * wp[a]
                                                       + nval * (gdd * wp[a] * wp[b] + gd * wpq[a][b]))
                                            + hdd * wp[a] * wp[b] + hd * wpq[a][b];
                        double cval = 6.0 * pow(r0, alp3);
                        double tval = cval * pow(ww, -aexp), tp[3], tpq[3][3];
                        for (int a = 0; a < 3; a++) tp[a] = -aexp * tval * wp[a] / ww;
                        for (int a = 0; a < 3; a++)
                            for (int b = 0; b < 3; b++)
                                tpq[a][b] = aexp * (aexp + 1.0) * tval * wp[a] * wp[b] / (ww * ww)
                                          - aexp * tval * wpq[a][b] / ww;
                        double fd = 1.0 / (1.0 + tval), fdp[3], fdpq[3][3];
                        for (int a = 0; a < 3; a++) fdp[a] = -tp[a] * fd * fd;
                        for (int a = 0; a < 3; a++)
                            for (int b = 0; b < 3; b++)
                                fdpq[a][b] = -tpq[a][b] * fd * fd + 2.0 * tp[a] * tp[b] * fd * fd * fd;
                        double av = ang * fd, ap[3], apq[3][3];
                        for (int a = 0; a < 3; a++) ap[a] = angp[a] * fd + ang * fdp[a];
                        for (int a = 0; a < 3; a++)
                            for (int b = 0; b < 3; b++)
                                apq[a][b] = angpq[a][b] * fd + angp[a] * fdp[b] + angp[b] * fdp[a] + ang * fdpq[a][b];
                        double kv = sval * av, kp[3], kpq[3][3];
                        for (int a = 0; a < 3; a++) kp[a] = sp[a] * av + sval * ap[a];
                        for (int a = 0; a < 3; a++)
                            for (int b = 0; b < 3; b++)
                                kpq[a][b] = spq[a][b] * av + sp[a] * ap[b] + sp[b] * ap[a] + sval * apq[a][b];
                        double qv = sqrt(fabs(c6t[0] * c6t[1] * c6t[2])), qm[3], qmn[3][3];
                        for (int a = 0; a < 3; a++) qm[a] = 0.5 * qv / c6t[a];
                        for (int a = 0; a < 3; a++)
                            for (int b = 0; b < 3; b++)
                                qmn[a][b] = (a == b) ? -0.25 * qv / (c6t[a] * c6t[a]) : 0.25 * qv / (c6t[a] * c6t[b]);
                        double pref = p->s9 * triple;
                        int at[3] = {i, j, kk};
                        double grad[3][3][3];   /* [c][atom][pair] */
                        for (int a = 0; a < 3; a++)
                            for (int q = 0; q < 3; q++)
                                for (int c = 0; c < 3; c++) grad[c][a][q] = 2.0 * sigp[a][q] * vec[q][c];
                        double pq = pref * qv, gk[3][3][3], dg[3][3];
                        for (int a = 0; a < 3; a++)
                            for (int c = 0; c < 3; c++)
                                for (int q = 0; q < 3; q++) {
                                    double tmp = 0.0;
                                    for (int s = 0; s < 3; s++) tmp += kpq[s][q] * grad[c][a][s];
                                    gk[c][a][q] = pq * tmp;
                                }
                        for (int a = 0; a < 3; a++)
                            for (int b = 0; b < 3; b++) {
                                double tmp = 0.0;
                                for (int s = 0; s < 3; s++) tmp += kp[s] * sigp[a][s] * sigp[b][s];
                                dg[a][b] = 2.0 * pq * tmp;
                            }
                        for (int a = 0; a < 3; a++)
                            for (int b = 0; b < 3; b++)
                                for (int c = 0; c < 3; c++)
                                    for (int d = 0; d < 3; d++) {
                                        double tmp = 0.0;
                                        for (int q = 0; q < 3; q++) tmp += gk[c][a][q] * grad[d][b][q];
                                        if (c == d) tmp += dg[a][b];
                                        H[(size_t)(3 * at[a] + c) * n3 + 3 * at[b] + d] += tmp;
                                    }
                        double ec[3], ecc[3][3], euc[3][3], egr[3][3][3];
                        for (int a = 0; a < 3; a++) {
                            ec[a] = pref * qm[a] * kv;
                            for (int b = 0; b < 3; b++) {
                                ecc[a][b] = pref * qmn[a][b] * kv;
                                euc[b][a] = pref * qm[a] * kp[b];
                            }
                        }
                        for (int a = 0; a < 3; a++)
                            for (int c = 0; c < 3; c++)
                                for (int mm = 0; mm < 3; mm++) {
                                    double tmp = 0.0;
                                    for (int s = 0; s < 3; s++) tmp += euc[s][mm] * grad[c][a][s];
                                    egr[c][a][mm] = tmp;
                                }
                        int pat[3][2] = {{i, j}, {i, kk}, {j, kk}};
                        int nent = 0, ent_atom[6], ent_pair[6];
                        double ent_coef[6];
                        for (int q = 0; q < 3; q++) {
                            int a1 = pat[q][0], a2 = pat[q][1];
                            if (a1 != a2) {
                                ent_atom[nent] = a1; ent_pair[nent] = q;
                                ent_coef[nent++] = dc6dcn[(size_t)a1 * nat + a2];
                                ent_atom[nent] = a2; ent_pair[nent] = q;
                                ent_coef[nent++] = dc6dcn[(size_t)a2 * nat + a1];
                            } else {
                                ent_atom[nent] = a1; ent_pair[nent] = q;
                                ent_coef[nent++] = 2.0 * dc6dcn[(size_t)a1 * nat + a1];
                            }
                        }
                        for (int e = 0; e < nent; e++) {
                            dEdcn[ent_atom[e]] += ec[ent_pair[e]] * ent_coef[e];
                            for (int f = 0; f < nent; f++)
                                D[(size_t)ent_atom[e] * nat + ent_atom[f]] +=
                                    ecc[ent_pair[e]][ent_pair[f]] * ent_coef[e] * ent_coef[f];
                            for (int a = 0; a < 3; a++)
                                for (int c = 0; c < 3; c++)
                                    A[(size_t)(3 * at[a] + c) * nat + ent_atom[e]] += egr[c][a][ent_pair[e]] * ent_coef[e];
                        }
                        for (int q = 0; q < 3; q++) {
                            int a1 = pat[q][0], a2 = pat[q][1];
                            if (a1 != a2) {
                                D[(size_t)a1 * nat + a1] += ec[q] * d2c6dcn2[(size_t)a1 * nat + a2];
                                D[(size_t)a2 * nat + a2] += ec[q] * d2c6dcn2[(size_t)a2 * nat + a1];
                                D[(size_t)a1 * nat + a2] += ec[q] * d2c6dcnij[(size_t)a1 * nat + a2];
                                D[(size_t)a2 * nat + a1] += ec[q] * d2c6dcnij[(size_t)a1 * nat + a2];
                            } else {
                                D[(size_t)a1 * nat + a1] += ec[q] * (2.0 * d2c6dcn2[(size_t)a1 * nat + a1]
                                                                    + 2.0 * d2c6dcnij[(size_t)a1 * nat + a1]);
                            }
                        }
                    }
                }
            }
        }
    }
}

static void cn_hessian(int nat, const double *xyz, const int *id, const double *rcov, const double *trans,
                       int ntr, double cutoff, const double *dEdcn, double *H)
{
    /* add_coordination_number_hessian, ncoord.f90:230-306 */
    size_t n3 = 3 * (size_t)nat;
    double cutoff2 = cutoff * cutoff;
    for (int i = 0; i < nat; i++) {
        int izp = id[i];
        for (int j = 0; j < i; j++) {
            int jzp = id[j];
            double rc = rcov[izp] + rcov[jzp];
            double dEdcnij = dEdcn[i] + dEdcn[j];
            for (int t = 0; t < ntr; t++) {
                double v[3];
                for (int c = 0; c < 3; c++) v[c] = xyz[3 * i + c] - (xyz[3 * j + c] + trans[3 * t + c]);
                double r2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
                if (r2 > cutoff2 || r2 < 1.0e-12) continue;
                double r1 = sqrt(r2);
                double cf = 1.0 / (1.0 + exp(-KCN * (rc / r1 - 1.0)));
                double tmp = cf * (1.0 - cf);
                double dcf = -tmp * KCN * rc / r2;
                double d2cf = tmp * (1.0 - 2.0 * cf) * (KCN * rc) * (KCN * rc) / (r2 * r2)
                            + 2.0 * tmp * KCN * rc / (r2 * r1);
                for (int a = 0; a < 3; a++)
                    for (int b = 0; b < 3; b++) {
                        double blk = dEdcnij * (d2cf * v[a] * v[b] / r2 - dcf * v[a] * v[b] / (r2 * r1));
                        if (a == b) blk += dEdcnij * dcf / r1;
                        H[(3 * i + a) * n3 + 3 * i + b] += blk;
                        H[(3 * j + a) * n3 + 3 * j + b] += blk;
                        H[(3 * i + a) * n3 + 3 * j + b] -= blk;
                        H[(3 * j + a) * n3 + 3 * i + b] -= blk;
                    }
            }
        }
    }
}

int oracle_get_dispersion_hessian(int nat, const int *numbers, const double *xyz, const double *lattice,
                                  const int *periodic, const int *ghost, const oracle_param *param,
                                  const oracle_cutoff *cutoff, int part, int nparts, double *hessian)
{
    /* get_dispersion_hessian, disp.f90:236-308 */
    if (param->damping < ORACLE_RATIONAL || param->damping > ORACLE_Z) return 4;
    model_t m;
    if (model_new(&m, nat, numbers, ghost)) return 1;
    double zero[9] = {0};
    int per0[3] = {0, 0, 0};
    const double *lat = lattice ? lattice : zero;
    const int *per = periodic ? periodic : per0;
    int mref = m.mref, ntr;
    size_t n = (size_t)(nat > 0 ? nat : 1), n3 = 3 * n, nn = n * n;
    double *cn = malloc(sizeof(double) * n);
    double *B = malloc(sizeof(double) * n3 * n);
    double *trans = lattice_points(lat, per, cutoff->cn, &ntr);
    cn_with_derivs(nat, xyz, m.id, m.rcov, trans, ntr, cutoff->cn, cn, B);
    free(trans);
    double *gw = malloc(sizeof(double) * n * mref), *dgw = malloc(sizeof(double) * n * mref);
    double *d2gw = malloc(sizeof(double) * n * mref);
    weight_references2(&m, nat, cn, gw, dgw, d2gw);
    double *c6 = malloc(sizeof(double) * nn), *dc6 = malloc(sizeof(double) * nn);
    double *d2c6 = malloc(sizeof(double) * nn), *d2c6ij = malloc(sizeof(double) * nn);
    get_atomic_c6_2(&m, nat, gw, dgw, d2gw, c6, dc6, d2c6, d2c6ij);
    double *dEdcn = calloc(n, sizeof(double));
    double *A = calloc(n3 * n, sizeof(double));
    double *D = calloc(nn, sizeof(double));
    memset(hessian, 0, sizeof(double) * 9 * (size_t)nat * nat);
    trans = lattice_points(lat, per, cutoff->disp2, &ntr);
    hessian2(&m, param, nat, xyz, trans, ntr, cutoff->disp2, cutoff->width2, c6, dc6, d2c6, d2c6ij, hessian, dEdcn,
             A, D, part, nparts);
    free(trans);
    trans = lattice_points(lat, per, cutoff->disp3, &ntr);
    hessian3(&m, param, nat, xyz, trans, ntr, cutoff->disp3, cutoff->width3, c6, dc6, d2c6, d2c6ij, hessian, dEdcn,
             A, D, part, nparts);
    free(trans);
    trans = lattice_points(lat, per, cutoff->cn, &ntr);
    cn_hessian(nat, xyz, m.id, m.rcov, trans, ntr, cutoff->cn, dEdcn, hessian);
    free(trans);
    /* H += A B^T + B A^T + B D B^T (disp.f90:299-301) */
    size_t N3 = 3 * (size_t)nat;
    double *DB = malloc(sizeof(double) * n * n3);   /* D B^T: [N][3N] */
    for (int k = 0; k < nat; k++)
        for (size_t b = 0; b < N3; b++) {
            double s = 0.0;
            for (int l = 0; l < nat; l++) s += D[(size_t)k * nat + l] * B[b * nat + l];
            DB[(size_t)k * N3 + b] = s;
        }
    for (size_t a = 0; a < N3; a++)
        for (size_t b = 0; b < N3; b++) {
            double s = 0.0;
            for (int k = 0; k < nat; k++)
                s += A[a * nat + k] * B[b * nat + k] + B[a * nat + k] * A[b * nat + k] + B[a * nat + k] * DB[(size_t)k * N3 + b];
            hessian[a * N3 + b] += s;
        }
    free(DB); free(cn); free(B); free(gw); free(dgw); free(d2gw); free(c6); free(dc6); free(d2c6); free(d2c6ij);
    free(dEdcn); free(A); free(D);
    model_free(&m);
    return 0;
}

static int pipeline(int nat, const int *numbers, const double *xyz, const double *lattice,
                    const int *periodic, const int *ghost, const oracle_param *param,
                    const oracle_cutoff *cutoff, int part, int nparts, oracle_reducer reduce, void *user,
                    double *energy, double *energies, double *gradient, double *sigma, double *cn_out,
                    double *dEdcn_out)
{
    /* get_dispersion_atomic_v2, disp.f90:56-185, and the scalar sum at :397.
     * With a reducer, the CN loop is partitioned and the CN and dE/dCN are
     * summed over the parts before use (disp.f90:120-126,166-171), and the
     * atom-resolved energies, gradient and virial afterwards
     * (get_dispersion_mpi_atomic, mpi.f90). */
    if (param->damping < ORACLE_RATIONAL || param->damping > ORACLE_Z) return 4;
    model_t m;
    if (model_new(&m, nat, numbers, ghost)) return 1;
    double zero[9] = {0};
    int per0[3] = {0, 0, 0};
    const double *lat = lattice ? lattice : zero;
    const int *per = periodic ? periodic : per0;
    int grad = gradient != NULL || sigma != NULL;
    int mref = m.mref;
    int threebody = fabs(param->s9) >= EPS;
    int ntr;
    int cn_part = reduce ? part : 0, cn_nparts = reduce ? nparts : 1;

    double *cn = malloc(sizeof(double) * (nat > 0 ? nat : 1));
    double *trans = lattice_points(lat, per, cutoff->cn, &ntr);
    partitioned_cn(nat, xyz, m.id, m.rcov, trans, ntr, cutoff->cn, cn, cn_part, cn_nparts);
    free(trans);
    if (reduce && reduce(cn, nat, user)) {
        free(cn);
        model_free(&m);
        return 2;
    }

    double *gwvec = malloc(sizeof(double) * (size_t)(nat > 0 ? nat : 1) * mref);
    double *gwdcn = grad ? malloc(sizeof(double) * (size_t)(nat > 0 ? nat : 1) * mref) : NULL;
    weight_references(&m, nat, cn, gwvec, gwdcn);

    size_t nn = (size_t)nat * nat;
    double *c6 = malloc(sizeof(double) * (nn > 0 ? nn : 1));
    double *dc6dcn = grad ? malloc(sizeof(double) * (nn > 0 ? nn : 1)) : NULL;
    if (threebody)
        get_atomic_c6(&m, nat, gwvec, gwdcn, c6, dc6dcn, 0, 1);
    else
        get_atomic_c6(&m, nat, gwvec, gwdcn, c6, dc6dcn, part, nparts);

    double *en = calloc(nat > 0 ? nat : 1, sizeof(double));
    double *dEdcn = grad ? calloc(nat > 0 ? nat : 1, sizeof(double)) : NULL;
    double *gl = grad ? calloc(3 * (size_t)(nat > 0 ? nat : 1), sizeof(double)) : NULL;
    double sl[9] = {0};

    trans = lattice_points(lat, per, cutoff->disp2, &ntr);
    dispersion2(&m, param, nat, xyz, trans, ntr, cutoff->disp2, cutoff->width2, c6, dc6dcn,
                en, dEdcn, gl, sl, part, nparts);
    free(trans);
    trans = lattice_points(lat, per, cutoff->disp3, &ntr);
    dispersion3(&m, param, nat, xyz, trans, ntr, cutoff->disp3, cutoff->width3, c6, dc6dcn,
                en, dEdcn, gl, sl, part, nparts);
    free(trans);
    int rc = 0;
    if (grad) {
        if (reduce && reduce(dEdcn, nat, user)) rc = 2;
        if (dEdcn_out)
            for (int i = 0; i < nat; i++) dEdcn_out[i] = dEdcn[i];
        trans = lattice_points(lat, per, cutoff->cn, &ntr);
        add_cn_derivs(nat, xyz, m.id, m.rcov, trans, ntr, cutoff->cn, dEdcn, gl, sl, cn_part, cn_nparts);
        free(trans);
    }
    if (reduce && rc == 0) {
        /* one fused sum of [energies | gradient | virial] */
        size_t len = (size_t)nat + (grad ? 3 * (size_t)nat + 9 : 0);
        double *buf = malloc(sizeof(double) * (len > 0 ? len : 1));
        memcpy(buf, en, sizeof(double) * nat);
        if (grad) {
            memcpy(buf + nat, gl, sizeof(double) * 3 * nat);
            memcpy(buf + 4 * (size_t)nat, sl, sizeof(double) * 9);
        }
        if (reduce(buf, (int)len, user)) rc = 2;
        memcpy(en, buf, sizeof(double) * nat);
        if (grad) {
            memcpy(gl, buf + nat, sizeof(double) * 3 * nat);
            memcpy(sl, buf + 4 * (size_t)nat, sizeof(double) * 9);
        }
        free(buf);
    }
    if (grad) {
        if (gradient) memcpy(gradient, gl, sizeof(double) * 3 * nat);
        if (sigma) memcpy(sigma, sl, sizeof(double) * 9);
    }
    double e = 0.0;
    for (int i = 0; i < nat; i++) e += en[i];
    if (energy) *energy = e;
    if (energies) memcpy(energies, en, sizeof(double) * nat);
    if (cn_out) memcpy(cn_out, cn, sizeof(double) * nat);

    free(cn); free(gwvec); free(gwdcn); free(c6); free(dc6dcn);
    free(en); free(dEdcn); free(gl);
    model_free(&m);
    return rc;
}

int oracle_get_dispersion(int nat, const int *numbers, const double *xyz,
                          const double *lattice, const int *periodic, const int *ghost,
                          const oracle_param *param, const oracle_cutoff *cutoff,
                          int part, int nparts, double *energy, double *energies,
                          double *gradient, double *sigma, double *cn_out, double *dEdcn_out)
{
    return pipeline(nat, numbers, xyz, lattice, periodic, ghost, param, cutoff, part, nparts, NULL, NULL,
                    energy, energies, gradient, sigma, cn_out, dEdcn_out);
}

int oracle_get_dispersion_reduced(int nat, const int *numbers, const double *xyz,
                                  const double *lattice, const int *periodic, const int *ghost,
                                  const oracle_param *param, const oracle_cutoff *cutoff,
                                  int part, int nparts, oracle_reducer reduce, void *user,
                                  double *energy, double *energies, double *gradient, double *sigma)
{
    if (!reduce) return 3;
    return pipeline(nat, numbers, xyz, lattice, periodic, ghost, param, cutoff, part, nparts, reduce, user,
                    energy, energies, gradient, sigma, NULL, NULL);
}
