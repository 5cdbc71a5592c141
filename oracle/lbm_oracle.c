/*
 * lbm_oracle.c -- FP64 CPU restatement of the reference's family-B D3Q19
 * acoustic solver.  TEST INFRASTRUCTURE ONLY (see lbm_oracle.h).
 *
 * Layout and arithmetic follow the reference one to one so that results are
 * bit-identical where the reference defines them:
 *   - AoS populations f[idx*19+q], idx = i + j*nx_t + k*nx_t*ny_t with a
 *     one-cell halo (06:206-209, 06:361-371);
 *   - every FP64 expression keeps the reference's operand order (feq 06:286-291,
 *     macro_at 06:545-568, the NSCBC ghost formulas 06:684-835, the BGK step
 *     06:906-972, the source 06:576-667, the mask/sponge 06:453-532 and the
 *     heightmap ray cast 06:144-192).  Compile with -ffp-contract=off.
 */
#include "lbm_oracle.h"

#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define Q 19
#define SOLID 1
#define FLUID 0

static const double CS2 = 1.0 / 3.0;                  /* 06:17 */
static const double CS = 0.57735026918962576451;      /* 06:18 */
static const double PI_ = 3.14159265358979323846;     /* 06:19 */

/* Family-B velocity order (06:21-23) and weights (06:25-31). */
static const int EX[Q] = {0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1, 0, 0, 0, 0};
static const int EY[Q] = {0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1};
static const int EZ[Q] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1};
static const double W[Q] = {1.0 / 3.0,
                            1.0 / 18.0, 1.0 / 18.0, 1.0 / 18.0, 1.0 / 18.0, 1.0 / 18.0, 1.0 / 18.0,
                            1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0,
                            1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0};

typedef struct { double x, y, z; } pt3;
typedef struct { pt3 v1, v2, v3, mn, mx; } tri_t;

typedef struct
{
    lbm_source s;
    double* table;   /* owned copy for LBM_WAVE_TABLE */
    double cx, cy, cz;
} src_t;

struct orc_handle
{
    lbm_config cfg;
    int inv_q[Q];
    int NXg, NYg, NZg, nx, ny, nz, nx_t, ny_t, nz_t;
    size_t Nloc;
    double dt;
    double *f_curr, *f_next, *rho, *sponge, *gH;
    double *tau_a, *field_a;   /* scheme A: per-cell tau (ramp sponge) and source weight */
    double *blend_xy, *field_xy;   /* scheme A: caller's per-column blend strengths, source weights */
    unsigned char* mask;
    int mask_override;
    /* geometry (GeometryEngine 06:60-193) */
    tri_t* tris;
    int ntris;
    pt3 gmin, gmax;
    double cellW, cellH;
    int* bin_start;   /* 200*200+1 CSR offsets */
    int* bin_items;
    /* sources / probes */
    src_t* srcs;
    int nsrc;
    int nprobe;
    double* probe_xyz;
    long* probe_idx;   /* -1: not owned */
    double* series;    /* [steps][nprobe] */
    long steps_rec, steps_cap;
    long step;         /* time steps taken by orc_step */
};

static inline size_t loc(const orc_handle* h, int i, int j, int k)
{
    return (size_t)i + (size_t)j * (size_t)h->nx_t + (size_t)k * (size_t)h->nx_t * (size_t)h->ny_t;
}

/* 06:286-291 */
static inline double feq(int k, double r, double ux, double uy, double uz)
{
    double cu = EX[k] * ux + EY[k] * uy + EZ[k] * uz;
    double u2 = ux * ux + uy * uy + uz * uz;
    return W[k] * r * (1.0 + 3.0 * cu + 4.5 * cu * cu - 1.5 * u2);
}

static double dmin(double a, double b) { return b < a ? b : a; }
static double dmax(double a, double b) { return a < b ? b : a; }
static double min3(double a, double b, double c) { return dmin(dmin(a, b), c); }
static double max3(double a, double b, double c) { return dmax(dmax(a, b), c); }

void orc_set_threads(int n) { omp_set_num_threads(n); }

orc_handle* orc_create(const lbm_config* cfg)
{
    orc_handle* h = (orc_handle*)calloc(1, sizeof(orc_handle));
    h->cfg = *cfg;
    /* inv_q as computed in LBMSolver::init (06:301-312) */
    for (int i = 0; i < Q; ++i)
    {
        h->inv_q[i] = 0;
        for (int j = 0; j < Q; ++j)
            if (EX[i] == -EX[j] && EY[i] == -EY[j] && EZ[i] == -EZ[j]) { h->inv_q[i] = j; break; }
    }
    h->gmin.x = h->gmin.y = h->gmin.z = 1e30;
    h->gmax.x = h->gmax.y = h->gmax.z = -1e30;
    h->cellW = h->cellH = 1.0;
    return h;
}

void orc_destroy(orc_handle* h)
{
    if (!h) return;
    free(h->f_curr); free(h->f_next); free(h->rho); free(h->sponge); free(h->gH); free(h->mask);
    free(h->tau_a); free(h->field_a); free(h->blend_xy); free(h->field_xy);
    free(h->tris); free(h->bin_start); free(h->bin_items);
    for (int i = 0; i < h->nsrc; ++i) free(h->srcs[i].table);
    free(h->srcs); free(h->probe_xyz); free(h->probe_idx); free(h->series);
    free(h);
}

/* ---------------------------------------------------------------- geometry */

/* GeometryEngine::buildGrid (06:113-142) with a 200x200 bin grid. */
static void build_grid(orc_handle* h)
{
    const int R = 200, C = 200;
    free(h->bin_start); free(h->bin_items);
    h->bin_start = NULL; h->bin_items = NULL;
    if (h->ntris == 0) return;
    h->cellW = (h->gmax.x - h->gmin.x) / R;
    h->cellH = (h->gmax.y - h->gmin.y) / C;
    if (h->cellW < 1e-9) h->cellW = 1.0;
    if (h->cellH < 1e-9) h->cellH = 1.0;
    int* cnt = (int*)calloc((size_t)R * C + 1, sizeof(int));
    int* rr = (int*)malloc((size_t)h->ntris * 4 * sizeof(int));
    for (int i = 0; i < h->ntris; ++i)
    {
        const tri_t* t = &h->tris[i];
        int r1 = (int)((t->mn.x - h->gmin.x) / h->cellW);
        int r2 = (int)((t->mx.x - h->gmin.x) / h->cellW);
        int c1 = (int)((t->mn.y - h->gmin.y) / h->cellH);
        int c2 = (int)((t->mx.y - h->gmin.y) / h->cellH);
        r1 = r1 < 0 ? 0 : (r1 > R - 1 ? R - 1 : r1);
        r2 = r2 < 0 ? 0 : (r2 > R - 1 ? R - 1 : r2);
        c1 = c1 < 0 ? 0 : (c1 > C - 1 ? C - 1 : c1);
        c2 = c2 < 0 ? 0 : (c2 > C - 1 ? C - 1 : c2);
        rr[4 * i] = r1; rr[4 * i + 1] = r2; rr[4 * i + 2] = c1; rr[4 * i + 3] = c2;
        for (int r = r1; r <= r2; ++r)
            for (int c = c1; c <= c2; ++c) cnt[r * C + c + 1]++;
    }
    for (int b = 0; b < R * C; ++b) cnt[b + 1] += cnt[b];
    h->bin_start = cnt;
    h->bin_items = (int*)malloc((size_t)(cnt[R * C] > 0 ? cnt[R * C] : 1) * sizeof(int));
    int* fill = (int*)calloc((size_t)R * C, sizeof(int));
    for (int i = 0; i < h->ntris; ++i)
        for (int r = rr[4 * i]; r <= rr[4 * i + 1]; ++r)
            for (int c = rr[4 * i + 2]; c <= rr[4 * i + 3]; ++c)
                h->bin_items[cnt[r * C + c] + fill[r * C + c]++] = i;
    free(fill);
    free(rr);
}

/* GeometryEngine::getGroundHeight (06:144-192): highest hit of the down ray. */
static double ground_height(const orc_handle* h, double x, double y)
{
    const int R = 200, C = 200;
    if (h->ntris == 0) return -1e30;
    if (x < h->gmin.x || x > h->gmax.x || y < h->gmin.y || y > h->gmax.y) return -1e30;
    int r = (int)((x - h->gmin.x) / h->cellW);
    int c = (int)((y - h->gmin.y) / h->cellH);
    if (r < 0 || r >= R || c < 0 || c >= C) return -1e30;
    const int b0 = h->bin_start[r * C + c], b1 = h->bin_start[r * C + c + 1];
    if (b0 == b1) return -1e30;
    const pt3 ro = {x, y, 10000.0};
    const pt3 rd = {0.0, 0.0, -1.0};
    double maxZ = -1e30;
    for (int b = b0; b < b1; ++b)
    {
        const tri_t* tri = &h->tris[h->bin_items[b]];
        if (tri->mx.x < x - 1e-6 || tri->mn.x > x + 1e-6) continue;
        if (tri->mx.y < y - 1e-6 || tri->mn.y > y + 1e-6) continue;
        const double EPS = 1e-9;
        pt3 e1 = {tri->v2.x - tri->v1.x, tri->v2.y - tri->v1.y, tri->v2.z - tri->v1.z};
        pt3 e2 = {tri->v3.x - tri->v1.x, tri->v3.y - tri->v1.y, tri->v3.z - tri->v1.z};
        pt3 hh = {rd.y * e2.z - rd.z * e2.y, rd.z * e2.x - rd.x * e2.z, rd.x * e2.y - rd.y * e2.x};
        double a = e1.x * hh.x + e1.y * hh.y + e1.z * hh.z;
        if (fabs(a) < EPS) continue;
        double f = 1.0 / a;
        pt3 s = {ro.x - tri->v1.x, ro.y - tri->v1.y, ro.z - tri->v1.z};
        double u = f * (s.x * hh.x + s.y * hh.y + s.z * hh.z);
        if (u < 0.0 || u > 1.0) continue;
        pt3 q = {s.y * e1.z - s.z * e1.y, s.z * e1.x - s.x * e1.z, s.x * e1.y - s.y * e1.x};
        double v = f * (rd.x * q.x + rd.y * q.y + rd.z * q.z);
        if (v < 0.0 || (u + v) > 1.0) continue;
        double t = f * (e2.x * q.x + e2.y * q.y + e2.z * q.z);
        if (t > EPS)
        {
            double hitZ = ro.z + t * rd.z;
            if (hitZ > maxZ) maxZ = hitZ;
        }
    }
    return maxZ;
}

static void add_triangle(orc_handle* h, int i, const float* v, double scale, double sx, double sy, double sz)
{
    tri_t* t = &h->tris[i];
    /* GeometryEngine::load (06:90-106) */
    t->v1.x = v[0] * scale + sx; t->v1.y = v[1] * scale + sy; t->v1.z = v[2] * scale + sz;
    t->v2.x = v[3] * scale + sx; t->v2.y = v[4] * scale + sy; t->v2.z = v[5] * scale + sz;
    t->v3.x = v[6] * scale + sx; t->v3.y = v[7] * scale + sy; t->v3.z = v[8] * scale + sz;
    t->mn.x = min3(t->v1.x, t->v2.x, t->v3.x);
    t->mn.y = min3(t->v1.y, t->v2.y, t->v3.y);
    t->mn.z = min3(t->v1.z, t->v2.z, t->v3.z);
    t->mx.x = max3(t->v1.x, t->v2.x, t->v3.x);
    t->mx.y = max3(t->v1.y, t->v2.y, t->v3.y);
    t->mx.z = max3(t->v1.z, t->v2.z, t->v3.z);
    h->gmin.x = dmin(h->gmin.x, t->mn.x); h->gmin.y = dmin(h->gmin.y, t->mn.y); h->gmin.z = dmin(h->gmin.z, t->mn.z);
    h->gmax.x = dmax(h->gmax.x, t->mx.x); h->gmax.y = dmax(h->gmax.y, t->mx.y); h->gmax.z = dmax(h->gmax.z, t->mx.z);
}

int orc_set_geometry_triangles(orc_handle* h, const float* tris, int ntris, double scale, double sx,
                               double sy, double sz)
{
    free(h->tris);
    h->tris = (tri_t*)calloc((size_t)(ntris > 0 ? ntris : 1), sizeof(tri_t));
    h->ntris = ntris;
    h->gmin.x = h->gmin.y = h->gmin.z = 1e30;
    h->gmax.x = h->gmax.y = h->gmax.z = -1e30;
    for (int i = 0; i < ntris; ++i) add_triangle(h, i, tris + 9 * (size_t)i, scale, sx, sy, sz);
    build_grid(h);
    return LBM_OK;
}

int orc_set_geometry_stl(orc_handle* h, const char* path, double scale, double sx, double sy, double sz)
{
    FILE* fp = fopen(path, "rb");
    if (!fp)
    {
        orc_set_geometry_triangles(h, NULL, 0, scale, sx, sy, sz);
        return LBM_WARN_STL_NOT_LOADED;
    }
    char header[80];
    uint32_t n = 0;
    if (fread(header, 1, 80, fp) != 80 || fread(&n, 4, 1, fp) != 1) n = 0;
    float* v = (float*)calloc((size_t)(n ? n : 1) * 9, sizeof(float));
    for (uint32_t i = 0; i < n; ++i)
    {
        unsigned char rec[50];
        memset(rec, 0, sizeof rec);
        size_t got = fread(rec, 1, 50, fp);
        (void)got;
        memcpy(v + 9 * (size_t)i, rec + 12, 36);
    }
    fclose(fp);
    orc_set_geometry_triangles(h, v, (int)n, scale, sx, sy, sz);
    free(v);
    return LBM_OK;
}

static double* copy_xy(const orc_handle* h, const double* v)
{
    const lbm_config* c = &h->cfg;
    const size_t n = (size_t)(int)((c->x_max - c->x_min) / c->dx + 0.5) * (size_t)(int)((c->y_max - c->y_min) / c->dx + 0.5);
    double* out = (double*)malloc(n * sizeof(double));
    if (out) memcpy(out, v, n * sizeof(double));
    return out;
}

int orc_set_blend_xy(orc_handle* h, const double* s_xy)
{
    free(h->blend_xy);
    h->blend_xy = copy_xy(h, s_xy);
    return h->blend_xy ? LBM_OK : LBM_ERR_OUT_OF_MEMORY;
}

int orc_set_field_xy(orc_handle* h, const double* w_xy)
{
    free(h->field_xy);
    h->field_xy = copy_xy(h, w_xy);
    return h->field_xy ? LBM_OK : LBM_ERR_OUT_OF_MEMORY;
}

int orc_set_mask(orc_handle* h, const unsigned char* mask)
{
    if (!h->mask) return LBM_ERR_STATE;
    memcpy(h->mask, mask, h->Nloc);
    h->mask_override = 1;
    return LBM_OK;
}

/* ---------------------------------------------------------- sources/probes */

int orc_add_source(orc_handle* h, const lbm_source* src)
{
    h->srcs = (src_t*)realloc(h->srcs, (size_t)(h->nsrc + 1) * sizeof(src_t));
    src_t* s = &h->srcs[h->nsrc++];
    memset(s, 0, sizeof *s);
    s->s = *src;
    if (src->waveform == LBM_WAVE_TABLE && src->table_len > 0)
    {
        s->table = (double*)malloc((size_t)src->table_len * sizeof(double));
        memcpy(s->table, src->table, (size_t)src->table_len * sizeof(double));
    }
    s->s.table = s->table;
    return LBM_OK;
}

int orc_set_probes(orc_handle* h, const double* xyz, int n)
{
    free(h->probe_xyz);
    h->probe_xyz = (double*)malloc((size_t)(n > 0 ? n : 1) * 3 * sizeof(double));
    memcpy(h->probe_xyz, xyz, (size_t)n * 3 * sizeof(double));
    h->nprobe = n;
    return LBM_OK;
}

/* ---------------------------------------------------------------- init */

static void halo_rules(orc_handle* h);

static void init_domain(orc_handle* h)
{
    const lbm_config* c = &h->cfg;
    const double dx = c->dx;
    const double sponge_w = c->sponge_width * dx;   /* 06:455 */
    const double strength = c->sponge_strength;     /* 06:456 */
    const double sky_z = c->sky_z;                  /* 06:458 */
    const unsigned sf = c->sponge_faces;

    /* 06:460-467 */
    #pragma omp parallel for collapse(2)
    for (int j = 0; j < h->ny_t; ++j)
        for (int i = 0; i < h->nx_t; ++i)
        {
            double x = c->x_min + ((i - 1) + 0.5) * dx;
            double y = c->y_min + ((j - 1) + 0.5) * dx;
            h->gH[(size_t)j * h->nx_t + (size_t)i] = ground_height(h, x, y);
        }

    /* 06:469-507 */
    #pragma omp parallel for collapse(2)
    for (int k = 0; k < h->nz_t; ++k)
        for (int j = 0; j < h->ny_t; ++j)
            for (int i = 0; i < h->nx_t; ++i)
            {
                size_t idx = loc(h, i, j, k);
                double x = c->x_min + ((i - 1) + 0.5) * dx;
                double y = c->y_min + ((j - 1) + 0.5) * dx;
                double z = c->z_min + ((k - 1) + 0.5) * dx;
                double gH = h->gH[(size_t)j * h->nx_t + (size_t)i];
                if (!h->mask_override)
                {
                    if (!c->use_geometry) h->mask[idx] = FLUID;
                    else h->mask[idx] = (z < gH) ? SOLID : FLUID;
                    if (z > sky_z) h->mask[idx] = FLUID;
                }
                double d = 1e30;
                if (sf & (1u << LBM_FACE_XLO)) d = dmin(d, x - c->x_min);
                if (sf & (1u << LBM_FACE_XHI)) d = dmin(d, c->x_max - x);
                if (sf & (1u << LBM_FACE_YLO)) d = dmin(d, y - c->y_min);
                if (sf & (1u << LBM_FACE_YHI)) d = dmin(d, c->y_max - y);
                if (sf & (1u << LBM_FACE_ZLO)) d = dmin(d, z - c->z_min);
                if (sf & (1u << LBM_FACE_ZHI)) d = dmin(d, c->z_max - z);
                if (d < sponge_w)
                {
                    double r = (sponge_w - d) / sponge_w;
                    h->sponge[idx] = strength * r * r;
                }
                else
                {
                    h->sponge[idx] = 0.0;
                }
            }

    if (!h->mask_override) halo_rules(h);
    /* periodic z (01:105-107): the halo planes are the opposite planes, also
       for a caller's mask */
    if (c->face_bc[LBM_FACE_ZLO] == LBM_BC_PERIODIC)
        for (int j = 0; j <= h->ny + 1; ++j)
            for (int i = 0; i <= h->nx + 1; ++i)
            {
                h->mask[loc(h, i, j, 0)] = h->mask[loc(h, i, j, h->nz)];
                h->mask[loc(h, i, j, h->nz + 1)] = h->mask[loc(h, i, j, 1)];
            }
}

/* Halo rules (06:509-531): x faces, then y faces, then z faces. */
static void halo_rules(orc_handle* h)
{
    const lbm_config* c = &h->cfg;
    const unsigned char mx0 = c->face_bc[LBM_FACE_XLO] == LBM_BC_WALL ? SOLID : FLUID;
    const unsigned char mx1 = c->face_bc[LBM_FACE_XHI] == LBM_BC_WALL ? SOLID : FLUID;
    const unsigned char my0 = c->face_bc[LBM_FACE_YLO] == LBM_BC_WALL ? SOLID : FLUID;
    const unsigned char my1 = c->face_bc[LBM_FACE_YHI] == LBM_BC_WALL ? SOLID : FLUID;
    const unsigned char mz0 = c->face_bc[LBM_FACE_ZLO] == LBM_BC_WALL ? SOLID : FLUID;
    const unsigned char mz1 = c->face_bc[LBM_FACE_ZHI] == LBM_BC_WALL ? SOLID : FLUID;
    for (int k = 0; k <= h->nz + 1; ++k)
        for (int j = 0; j <= h->ny + 1; ++j)
        {
            h->mask[loc(h, 0, j, k)] = mx0;
            h->mask[loc(h, h->nx + 1, j, k)] = mx1;
        }
    for (int k = 0; k <= h->nz + 1; ++k)
        for (int i = 0; i <= h->nx + 1; ++i)
        {
            h->mask[loc(h, i, 0, k)] = my0;
            h->mask[loc(h, i, h->ny + 1, k)] = my1;
        }
    for (int j = 0; j <= h->ny + 1; ++j)
        for (int i = 0; i <= h->nx + 1; ++i)
        {
            h->mask[loc(h, i, j, 0)] = mz0;
            h->mask[loc(h, i, j, h->nz + 1)] = mz1;
        }
}

static double source_value(const orc_handle* h, const src_t* s, double t);

/* ---------------------------------------------------------------- scheme A
 * The reference's family-A update (01-04): every population arriving at a
 * fluid cell is the post-collision value of the cell it left, relaxed with
 * that cell's tau; a population arriving from a SOLID cell is the
 * destination's own pre-collision value of the opposite direction; SOLID
 * cells are not updated (02:363-420, 03:402-441).  Family-A direction order
 * (02:15-19, 03:15-17). */
static const int EXA[Q] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
static const int EYA[Q] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1};
static const int EZA[Q] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1};
static const int INVA[Q] = {0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17};

static inline double feq_a(int q, double r, double ux, double uy, double uz)
{
    double cu = EXA[q] * ux + EYA[q] * uy + EZA[q] * uz;
    double u2 = ux * ux + uy * uy + uz * uz;
    return W[q] * r * (1.0 + 3.0 * cu + 4.5 * cu * cu - 1.5 * u2);
}

/* tau ramp (02:164-179, 03:148-160): d = whole cells to the nearest sponge
 * face (halo cells have d < 0), tau = tau + (max - tau) ((w - d) / w)^2 for
 * 0 <= d < w; source weights exp(-|x - s|^2 / (2 sigma^2)) at every cell
 * centre (02:181, 03:166-169); initial state feq(1, flow) (03:162-163). */
static void init_scheme_a(orc_handle* h)
{
    const lbm_config* c = &h->cfg;
    const unsigned sf = c->sponge_faces;
    const int w = (int)c->sponge_width;
    free(h->tau_a);
    free(h->field_a);   /* a second orc_init (after orc_set_mask) rebuilds both */
    h->tau_a = (double*)malloc(h->Nloc * sizeof(double));
    h->field_a = (double*)calloc(h->Nloc, sizeof(double));
    const src_t* fs = NULL;
    for (int i = 0; i < h->nsrc; ++i)
        if (h->srcs[i].s.injection == LBM_INJECT_FIELD) fs = &h->srcs[i];
    const double sig = fs ? fs->s.sigma_cells * c->dx : 1.0;
    #pragma omp parallel for collapse(2)
    for (int k = 0; k < h->nz_t; ++k)
        for (int j = 0; j < h->ny_t; ++j)
            for (int i = 0; i < h->nx_t; ++i)
            {
                const size_t idx = loc(h, i, j, k);
                const int gx = i - 1, gy = j - 1, gz = k - 1;
                int d = 1 << 30;
                if (sf & (1u << LBM_FACE_XLO)) d = gx < d ? gx : d;
                if (sf & (1u << LBM_FACE_XHI)) d = h->NXg - 1 - gx < d ? h->NXg - 1 - gx : d;
                if (sf & (1u << LBM_FACE_YLO)) d = gy < d ? gy : d;
                if (sf & (1u << LBM_FACE_YHI)) d = h->NYg - 1 - gy < d ? h->NYg - 1 - gy : d;
                if (sf & (1u << LBM_FACE_ZLO)) d = gz < d ? gz : d;
                if (sf & (1u << LBM_FACE_ZHI)) d = h->NZg - 1 - gz < d ? h->NZg - 1 - gz : d;
                double tau = c->tau;
                if (c->tau_sponge_max > 0 && d >= 0 && d < w)
                {
                    const double r = (double)(w - d) / w;
                    tau = c->tau + (c->tau_sponge_max - c->tau) * r * r;
                }
                h->tau_a[idx] = tau;
                if (fs)
                {
                    const double x = c->x_min + (gx + 0.5) * c->dx - fs->s.sx;
                    const double y = c->y_min + (gy + 0.5) * c->dx - fs->s.sy;
                    const double z = c->z_min + (gz + 0.5) * c->dx - fs->s.sz;
                    h->field_a[idx] = exp(-(x * x + y * y + z * z) / (2.0 * sig * sig));
                }
                /* a caller's per-column weights (nearest column for halo cells) */
                const int cx = gx < 0 ? 0 : (gx >= h->nx ? h->nx - 1 : gx);
                const int cy = gy < 0 ? 0 : (gy >= h->ny ? h->ny - 1 : gy);
                if (h->field_xy) h->field_a[idx] = h->field_xy[(size_t)cy * h->nx + cx];
                for (int q = 0; q < Q; ++q) h->f_curr[idx * Q + q] = feq_a(q, 1.0, c->flow[0], c->flow[1], c->flow[2]);
                if (c->sponge_blend)
                {
                    /* 01's sponge (01:207-225): distance into the layer per axis, the
                       largest of them, strength (dist / thickness)^2 */
                    const double th = c->sponge_width * c->dx;
                    const double x = c->x_min + (gx + 0.5) * c->dx;
                    const double y = c->y_min + (gy + 0.5) * c->dx;
                    const double z = c->z_min + (gz + 0.5) * c->dx;
                    double dist_x = 0.0, dist_y = 0.0, dist_z = 0.0;
                    if ((sf & (1u << LBM_FACE_XLO)) && x < c->x_min + th) dist_x = (c->x_min + th) - x;
                    else if ((sf & (1u << LBM_FACE_XHI)) && x > c->x_max - th) dist_x = x - (c->x_max - th);
                    if ((sf & (1u << LBM_FACE_YLO)) && y < c->y_min + th) dist_y = (c->y_min + th) - y;
                    else if ((sf & (1u << LBM_FACE_YHI)) && y > c->y_max - th) dist_y = y - (c->y_max - th);
                    if ((sf & (1u << LBM_FACE_ZLO)) && z < c->z_min + th) dist_z = (c->z_min + th) - z;
                    else if ((sf & (1u << LBM_FACE_ZHI)) && z > c->z_max - th) dist_z = z - (c->z_max - th);
                    double dist_max = dist_x > dist_y ? dist_x : dist_y;
                    dist_max = dist_z > dist_max ? dist_z : dist_max;
                    double sig = 0.0;
                    if (dist_max > 0.0)
                    {
                        const double r_ratio = dist_max / th;
                        sig = c->sponge_strength * r_ratio * r_ratio;
                    }
                    if (h->blend_xy && h->blend_xy[(size_t)cy * h->nx + cx] > sig) sig = h->blend_xy[(size_t)cy * h->nx + cx];
                    h->sponge[idx] = sig;
                }
            }
}

/* Halo fill of a scheme-A step: REST faces hold feq(1, 0) (02:227-360 at
 * MPI size 1), COPY faces take the nearest interior cell (03:175-237, x
 * faces first, then y, then z, each over the whole halo plane). */
static void halos_a(orc_handle* h)
{
    const lbm_config* c = &h->cfg;
    if (c->face_bc[0] == LBM_BC_COPY)
    {
        const int nxt = h->nx_t, nyt = h->ny_t, nzt = h->nz_t;
        for (int k = 0; k < nzt; ++k)
            for (int j = 0; j < nyt; ++j)
            {
                memcpy(&h->f_curr[loc(h, 0, j, k) * Q], &h->f_curr[loc(h, 1, j, k) * Q], Q * sizeof(double));
                memcpy(&h->f_curr[loc(h, h->nx + 1, j, k) * Q], &h->f_curr[loc(h, h->nx, j, k) * Q], Q * sizeof(double));
            }
        for (int k = 0; k < nzt; ++k)
            for (int i = 0; i < nxt; ++i)
            {
                memcpy(&h->f_curr[loc(h, i, 0, k) * Q], &h->f_curr[loc(h, i, 1, k) * Q], Q * sizeof(double));
                memcpy(&h->f_curr[loc(h, i, h->ny + 1, k) * Q], &h->f_curr[loc(h, i, h->ny, k) * Q], Q * sizeof(double));
            }
        for (int j = 0; j < nyt; ++j)
            for (int i = 0; i < nxt; ++i)
            {
                memcpy(&h->f_curr[loc(h, i, j, 0) * Q], &h->f_curr[loc(h, i, j, 1) * Q], Q * sizeof(double));
                memcpy(&h->f_curr[loc(h, i, j, h->nz + 1) * Q], &h->f_curr[loc(h, i, j, h->nz) * Q], Q * sizeof(double));
            }
        return;
    }
    orc_exchange_halos(h);   /* REST faces: feq(1,0); WALL halos are SOLID and never read */
    if (c->face_bc[LBM_FACE_ZLO] == LBM_BC_PERIODIC)
    {
        /* 01:286-299 at one rank: the rank is its own z neighbour, whole planes */
        const size_t plane = (size_t)h->nx_t * h->ny_t * Q;
        memcpy(&h->f_curr[loc(h, 0, 0, 0) * Q], &h->f_curr[loc(h, 0, 0, h->nz) * Q], plane * sizeof(double));
        memcpy(&h->f_curr[loc(h, 0, 0, h->nz + 1) * Q], &h->f_curr[loc(h, 0, 0, 1) * Q], plane * sizeof(double));
    }
}

/* One scheme-A step at step index s (time t = s dt). */
void orc_exchange_halos(orc_handle* h);

static void step_a(orc_handle* h, long s)
{
    const lbm_config* c = &h->cfg;
    const double t = s * h->dt;
    const src_t* fs = NULL;
    for (int i = 0; i < h->nsrc; ++i)
        if (h->srcs[i].s.injection == LBM_INJECT_FIELD) fs = &h->srcs[i];
    const double mass = fs ? source_value(h, fs, t) * h->dt * fs->s.gain : 0.0;
    const int force = fs && fs->s.field_mode == LBM_FIELD_FORCE;
    const int pre = fs && fs->s.field_mode == LBM_FIELD_PRE;
    const double fx = c->flow[0], fy = c->flow[1], fz = c->flow[2];
    if (pre)
    {
        /* 04:212-235: every population of every interior fluid cell, before the
           halo exchange and the step */
        #pragma omp parallel for collapse(2)
        for (int k = 1; k <= h->nz; ++k)
            for (int j = 1; j <= h->ny; ++j)
                for (int i = 1; i <= h->nx; ++i)
                {
                    const size_t idx = loc(h, i, j, k);
                    if (h->mask[idx] == SOLID) continue;
                    for (int q = 0; q < Q; ++q) h->f_curr[idx * Q + q] += W[q] * (h->field_a[idx] * mass);
                }
    }
    halos_a(h);
    const int nx = h->nx, ny = h->ny, nz = h->nz;
    #pragma omp parallel for collapse(2)
    for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i)
            {
                const size_t dst = loc(h, i, j, k);
                if (h->mask[dst] == SOLID) continue;
                double rho_new = 0.0;
                for (int q = 0; q < Q; ++q)
                {
                    const size_t src = loc(h, i - EXA[q], j - EYA[q], k - EZA[q]);
                    double fn;
                    if (h->mask[src] == SOLID)
                    {
                        fn = h->f_curr[dst * Q + INVA[q]];
                    }
                    else
                    {
                        double r = 0, ux = 0, uy = 0, uz = 0;
                        for (int p = 0; p < Q; ++p)
                        {
                            const double v = h->f_curr[src * Q + p];
                            r += v;
                            ux += v * EXA[p];
                            uy += v * EYA[p];
                            uz += v * EZA[p];
                        }
                        if (r > 1e-12)
                        {
                            ux /= r; uy /= r; uz /= r;
                        }
                        else
                        {
                            r = 1.0; ux = fx; uy = fy; uz = fz;
                        }
                        const double tau_s = h->tau_a[src];
                        const double fo = h->f_curr[src * Q + q];
                        fn = fo - (fo - feq_a(q, r, ux, uy, uz)) / tau_s;
                        if (force)
                        {
                            const double cu = EXA[q] * fx + EYA[q] * fy + EZA[q] * fz;
                            fn += W[q] * (h->field_a[src] * mass) * (1.0 + 3.0 * cu) * (1.0 - 0.5 / tau_s);
                        }
                        else if (fs && !pre)
                        {
                            fn += W[q] * (h->field_a[dst] * mass);
                        }
                        if (c->sponge_blend && h->sponge[dst] > 1e-6)
                        {
                            /* 01:343-347 */
                            const double sigma = h->sponge[dst];
                            fn = (1.0 - sigma) * fn + sigma * feq_a(q, 1.0, 0.0, 0.0, 0.0);
                        }
                    }
                    h->f_next[dst * Q + q] = fn;
                    rho_new += fn;
                }
                h->rho[dst] = rho_new;
            }
    double* tmp = h->f_curr;
    h->f_curr = h->f_next;
    h->f_next = tmp;
}

int orc_init(orc_handle* h)
{
    const lbm_config* c = &h->cfg;
    /* 06:332-334 */
    h->NXg = (int)((c->x_max - c->x_min) / c->dx + 0.5);
    h->NYg = (int)((c->y_max - c->y_min) / c->dx + 0.5);
    h->NZg = (int)((c->z_max - c->z_min) / c->dx + 0.5);
    h->nx = h->NXg; h->ny = h->NYg; h->nz = h->NZg;
    h->nx_t = h->nx + 2; h->ny_t = h->ny + 2; h->nz_t = h->nz + 2;
    h->Nloc = (size_t)h->nx_t * h->ny_t * h->nz_t;
    h->dt = (CS * c->dx) / c->c_phys;   /* UnitConverter::get_dt_phys 06:200-203 */
    if (c->dt > 0) h->dt = c->dt;

    int had_mask = h->mask != NULL && h->mask_override;
    unsigned char* keep = NULL;
    if (had_mask) { keep = h->mask; h->mask = NULL; }
    free(h->f_curr); free(h->f_next); free(h->rho); free(h->sponge); free(h->gH); free(h->mask);
    h->f_curr = (double*)malloc(h->Nloc * Q * sizeof(double));
    h->f_next = (double*)calloc(h->Nloc * Q, sizeof(double));
    h->rho = (double*)malloc(h->Nloc * sizeof(double));
    h->sponge = (double*)calloc(h->Nloc, sizeof(double));
    h->gH = (double*)malloc((size_t)h->nx_t * h->ny_t * sizeof(double));
    h->mask = keep ? keep : (unsigned char*)calloc(h->Nloc, 1);
    if (!h->f_curr || !h->f_next || !h->rho || !h->sponge || !h->gH || !h->mask) return LBM_ERR_OUT_OF_MEMORY;
    for (size_t i = 0; i < h->Nloc; ++i) h->rho[i] = 1.0;

    double feq0[Q];
    for (int q = 0; q < Q; ++q) feq0[q] = feq(q, 1.0, 0.0, 0.0, 0.0);
    #pragma omp parallel for
    for (long i = 0; i < (long)h->Nloc; ++i)
        for (int q = 0; q < Q; ++q) h->f_curr[(size_t)i * Q + q] = feq0[q];

    init_domain(h);
    if (c->scheme == LBM_SCHEME_A) init_scheme_a(h);

    int status = LBM_OK;
    free(h->probe_idx);
    h->probe_idx = (long*)malloc((size_t)(h->nprobe > 0 ? h->nprobe : 1) * sizeof(long));
    for (int p = 0; p < h->nprobe; ++p)
    {
        /* 06:415-437 */
        int gi = (int)floor((h->probe_xyz[3 * p] - c->x_min) / c->dx);
        int gj = (int)floor((h->probe_xyz[3 * p + 1] - c->y_min) / c->dx);
        int gk = (int)floor((h->probe_xyz[3 * p + 2] - c->z_min) / c->dx);
        h->probe_idx[p] = -1;
        if (gi >= 0 && gi < h->nx && gj >= 0 && gj < h->ny && gk >= 0 && gk < h->nz)
        {
            h->probe_idx[p] = (long)loc(h, gi + 1, gj + 1, gk + 1);
            if (h->mask[h->probe_idx[p]] == SOLID) status = LBM_WARN_PROBE_IN_SOLID;
        }
    }
    free(h->series);
    h->series = NULL;
    h->steps_rec = h->steps_cap = 0;
    h->step = 0;
    return status;
}

/* ---------------------------------------------------------------- source */

/* DroneSource::update (06:221-238) */
static void drone_update(src_t* s, double t)
{
    double dx = s->s.ex - s->s.sx, dy = s->s.ey - s->s.sy, dz = s->s.ez - s->s.sz;
    double dist_total = sqrt(dx * dx + dy * dy + dz * dz);
    if (dist_total < 1e-12 || s->s.speed < 1e-12)
    {
        s->cx = s->s.sx; s->cy = s->s.sy; s->cz = s->s.sz;
        return;
    }
    double travel_time = dist_total / s->s.speed;
    double r = t / travel_time;
    if (r > 1.0) r = 1.0;
    s->cx = s->s.sx + r * dx;
    s->cy = s->s.sy + r * dy;
    s->cz = s->s.sz + r * dz;
}

static double source_value(const orc_handle* h, const src_t* s, double t)
{
    const lbm_source* p = &s->s;
    switch (p->waveform)
    {
    case LBM_WAVE_GAUSS:   /* 06:579-581 */
        return p->amp * exp(-0.5 * pow((t - p->t0) / p->sigma_t, 2));
    case LBM_WAVE_SINE:    /* 08:543 */
        return p->amp * sin(2.0 * PI_ * p->freq * t);
    case LBM_WAVE_RICKER:
    {
        double a = PI_ * p->freq * (t - p->t0);
        a = a * a;
        return p->amp * (1.0 - 2.0 * a) * exp(-a);
    }
    case LBM_WAVE_TABLE:
    {
        long s_idx = lround(t / h->dt);
        if (s_idx < 0 || s_idx >= p->table_len) return 0.0;
        return p->amp * p->table[s_idx];
    }
    }
    return 0.0;
}

static int cell_in_grid(const orc_handle* h, int gi, int gj, int gk)
{
    return !(gi < 0 || gi >= h->NXg || gj < 0 || gj >= h->NYg || gk < 0 || gk >= h->NZg);
}

/* LBMSolver::apply_source (06:576-667; 08:540-628 for the sine), one source. */
static void apply_one_source(orc_handle* h, src_t* s, double t)
{
    if (s->s.injection == LBM_INJECT_FIELD) return;   /* scheme A: applied inside step_a */
    const lbm_config* c = &h->cfg;
    const double dt = h->dt;
    const double DX = c->dx;
    const double val = source_value(h, s, t);
    const double source_gain = s->s.gain;
    drone_update(s, t);

    if (s->s.injection == LBM_INJECT_TRILINEAR)
    {
        double fx = (s->cx - c->x_min) / DX - 0.5;
        double fy = (s->cy - c->y_min) / DX - 0.5;
        double fz = (s->cz - c->z_min) / DX - 0.5;
        int i0 = (int)floor(fx), j0 = (int)floor(fy), k0 = (int)floor(fz);
        double tx = fx - i0, ty = fy - j0, tz = fz - k0;
        double sumw = 0.0;
        for (int b = 0; b < 8; ++b)
        {
            int gi = i0 + (b & 1), gj = j0 + ((b >> 1) & 1), gk = k0 + (b >> 2);
            if (!cell_in_grid(h, gi, gj, gk)) continue;
            double ww = ((b & 1) ? tx : 1.0 - tx) * (((b >> 1) & 1) ? ty : 1.0 - ty) * ((b >> 2) ? tz : 1.0 - tz);
            if (h->mask[loc(h, gi + 1, gj + 1, gk + 1)] == FLUID) sumw += ww;
        }
        if (sumw < 1e-30) return;
        const double A = (val * dt * source_gain) / sumw;
        for (int b = 0; b < 8; ++b)
        {
            int gi = i0 + (b & 1), gj = j0 + ((b >> 1) & 1), gk = k0 + (b >> 2);
            if (!cell_in_grid(h, gi, gj, gk)) continue;
            size_t idx = loc(h, gi + 1, gj + 1, gk + 1);
            if (h->mask[idx] != FLUID) continue;
            double ww = ((b & 1) ? tx : 1.0 - tx) * (((b >> 1) & 1) ? ty : 1.0 - ty) * ((b >> 2) ? tz : 1.0 - tz);
            const double add = A * ww;
            for (int q = 0; q < Q; ++q) h->f_curr[idx * Q + q] += W[q] * add;
        }
        return;
    }

    const int R = s->s.radius;
    const double sigma_cells = s->s.sigma_cells;
    const double sigma2 = (sigma_cells * DX) * (sigma_cells * DX);
    const int ic = (int)floor((s->cx - c->x_min) / DX);
    const int jc = (int)floor((s->cy - c->y_min) / DX);
    const int kc = (int)floor((s->cz - c->z_min) / DX);
    if (ic < -R || ic >= h->NXg + R || jc < -R || jc >= h->NYg + R || kc < -R || kc >= h->NZg + R) return;

    double sumw = 0.0;
    for (int gk = kc - R; gk <= kc + R; ++gk)
        for (int gj = jc - R; gj <= jc + R; ++gj)
            for (int gi = ic - R; gi <= ic + R; ++gi)
            {
                if (!cell_in_grid(h, gi, gj, gk)) continue;
                const double x = c->x_min + (gi + 0.5) * DX;
                const double y = c->y_min + (gj + 0.5) * DX;
                const double z = c->z_min + (gk + 0.5) * DX;
                const double ddx = x - s->cx, ddy = y - s->cy, ddz = z - s->cz;
                const double r2 = ddx * ddx + ddy * ddy + ddz * ddz;
                const double ww = exp(-0.5 * r2 / sigma2);
                if (h->mask[loc(h, gi + 1, gj + 1, gk + 1)] == FLUID) sumw += ww;
            }
    if (sumw < 1e-30) return;
    const double A = (val * dt * source_gain) / sumw;
    for (int gk = kc - R; gk <= kc + R; ++gk)
        for (int gj = jc - R; gj <= jc + R; ++gj)
            for (int gi = ic - R; gi <= ic + R; ++gi)
            {
                if (!cell_in_grid(h, gi, gj, gk)) continue;
                const double x = c->x_min + (gi + 0.5) * DX;
                const double y = c->y_min + (gj + 0.5) * DX;
                const double z = c->z_min + (gk + 0.5) * DX;
                const double ddx = x - s->cx, ddy = y - s->cy, ddz = z - s->cz;
                const double r2 = ddx * ddx + ddy * ddy + ddz * ddz;
                const double ww = exp(-0.5 * r2 / sigma2);
                const size_t idx = loc(h, gi + 1, gj + 1, gk + 1);
                if (h->mask[idx] != FLUID) continue;
                const double add = A * ww;
                for (int q = 0; q < Q; ++q) h->f_curr[idx * Q + q] += W[q] * add;
            }
}

void orc_apply_source(orc_handle* h, double t)
{
    for (int i = 0; i < h->nsrc; ++i) apply_one_source(h, &h->srcs[i], t);
}

/* ---------------------------------------------------------------- halos */

/* LBMSolver::macro_at (06:545-568) */
static void macro_at(const orc_handle* h, size_t idx, double* r, double* ux, double* uy, double* uz)
{
    *r = *ux = *uy = *uz = 0.0;
    const size_t base = idx * Q;
    for (int q = 0; q < Q; ++q)
    {
        const double fq = h->f_curr[base + q];
        *r += fq;
        *ux += fq * EX[q];
        *uy += fq * EY[q];
        *uz += fq * EZ[q];
    }
    if (*r > 1e-30)
    {
        *ux /= *r; *uy /= *r; *uz /= *r;
    }
    else
    {
        *r = 1.0;
        *ux = *uy = *uz = 0.0;
    }
}

/* Ghost populations for one open-face cell from its interior neighbour
 * (06:689-707 pattern): axis 0/1/2, side 0 = low face, 1 = high face. */
static void nscbc_ghost(const orc_handle* h, size_t idxI, int axis, int side, double* out)
{
    double rI, u[3];
    macro_at(h, idxI, &rI, &u[0], &u[1], &u[2]);
    const double pI = CS2 * (rI - 1.0);
    double Wp, Wm, unB, pB;
    if (side == 0)
    {
        Wp = 0.0;
        Wm = u[axis] - pI / CS;
    }
    else
    {
        Wm = 0.0;
        Wp = u[axis] + pI / CS;
    }
    unB = 0.5 * (Wp + Wm);
    pB = 0.5 * CS * (Wp - Wm);
    const double rhoB = 1.0 + pB / CS2;
    double uB[3] = {u[0], u[1], u[2]};
    uB[axis] = unB;
    const size_t baseI = idxI * Q;
    for (int q = 0; q < Q; ++q)
    {
        const double feqI = feq(q, rI, u[0], u[1], u[2]);
        const double feqB = feq(q, rhoB, uB[0], uB[1], uB[2]);
        out[q] = feqB + (h->f_curr[baseI + q] - feqI);
    }
}

/* LBMSolver::exchange_halos (06:671-904) at MPI size 1: every halo cell is
 * rewritten from interior cells only, so the evaluation order of the faces
 * does not matter; edge/corner halo cells hold w_q. */
void orc_exchange_halos(orc_handle* h)
{
    const lbm_config* c = &h->cfg;
    const int nx = h->nx, ny = h->ny, nz = h->nz;
    double feq0[Q];
    for (int q = 0; q < Q; ++q) feq0[q] = feq(q, 1.0, 0.0, 0.0, 0.0);

    /* x faces: j 1..ny, k 1..nz (06:684-736, unpack 06:853-859) */
    for (int side = 0; side < 2; ++side)
    {
        const int nscbc = c->face_bc[LBM_FACE_XLO + side] == LBM_BC_NSCBC;
        const int ig = side ? nx + 1 : 0, ii = side ? nx : 1;
        #pragma omp parallel for
        for (int k = 1; k <= nz; ++k)
            for (int j = 1; j <= ny; ++j)
            {
                double g[Q];
                if (nscbc) nscbc_ghost(h, loc(h, ii, j, k), 0, side, g);
                else memcpy(g, feq0, sizeof g);
                double* dst = &h->f_curr[loc(h, ig, j, k) * Q];
                /* ghosts read only interior cells; writing in place is safe */
                for (int q = 0; q < Q; ++q) dst[q] = g[q];
            }
    }
    /* y faces: i 0..nx+1 (edges w_q), k 1..nz (06:738-802, unpack 06:875-881) */
    for (int side = 0; side < 2; ++side)
    {
        const int nscbc = c->face_bc[LBM_FACE_YLO + side] == LBM_BC_NSCBC;
        const int jg = side ? ny + 1 : 0, ji = side ? ny : 1;
        #pragma omp parallel for
        for (int k = 1; k <= nz; ++k)
            for (int i = 0; i <= nx + 1; ++i)
            {
                double g[Q];
                if (nscbc && i != 0 && i != nx + 1) nscbc_ghost(h, loc(h, i, ji, k), 1, side, g);
                else memcpy(g, feq0, sizeof g);
                double* dst = &h->f_curr[loc(h, i, jg, k) * Q];
                for (int q = 0; q < Q; ++q) dst[q] = g[q];
            }
    }
    /* z faces: all i, j (edges w_q) (06:804-835, unpack 06:897-903) */
    for (int side = 0; side < 2; ++side)
    {
        const int nscbc = c->face_bc[LBM_FACE_ZLO + side] == LBM_BC_NSCBC;
        const int kg = side ? nz + 1 : 0, ki = side ? nz : 1;
        #pragma omp parallel for
        for (int j = 0; j <= ny + 1; ++j)
            for (int i = 0; i <= nx + 1; ++i)
            {
                double g[Q];
                if (nscbc && i != 0 && i != nx + 1 && j != 0 && j != ny + 1)
                    nscbc_ghost(h, loc(h, i, j, ki), 2, side, g);
                else memcpy(g, feq0, sizeof g);
                double* dst = &h->f_curr[loc(h, i, j, kg) * Q];
                for (int q = 0; q < Q; ++q) dst[q] = g[q];
            }
    }
}

/* ---------------------------------------------------------------- step */

/* LBMSolver::step_collision_bgk (06:906-972) */
void orc_step_collision_bgk(orc_handle* h)
{
    const double omega = 1.0 / h->cfg.tau;
    const int nx = h->nx, ny = h->ny, nz = h->nz;
    #pragma omp parallel for collapse(2)
    for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i)
            {
                size_t dst = loc(h, i, j, k);
                double f_in[Q];
                for (int q = 0; q < Q; ++q)
                {
                    size_t src = loc(h, i - EX[q], j - EY[q], k - EZ[q]);
                    if (h->mask[src] == SOLID) f_in[q] = h->f_curr[dst * Q + h->inv_q[q]];
                    else f_in[q] = h->f_curr[src * Q + q];
                }
                if (h->mask[dst] == SOLID)
                {
                    for (int q = 0; q < Q; ++q) h->f_next[dst * Q + q] = f_in[q];
                    h->rho[dst] = 1.0;
                    continue;
                }
                double r = 0, jx = 0, jy = 0, jz = 0;
                for (int q = 0; q < Q; ++q)
                {
                    r += f_in[q];
                    jx += f_in[q] * EX[q];
                    jy += f_in[q] * EY[q];
                    jz += f_in[q] * EZ[q];
                }
                if (r <= 0.0) r = 1e-12;
                double ux = jx / r, uy = jy / r, uz = jz / r;
                h->rho[dst] = r;
                double sponge = h->sponge[dst];
                for (int q = 0; q < Q; ++q)
                {
                    double feq_q = feq(q, r, ux, uy, uz);
                    double f_post = f_in[q] - omega * (f_in[q] - feq_q);
                    if (sponge > 1e-12)
                    {
                        double feq0 = feq(q, 1.0, 0.0, 0.0, 0.0);
                        f_post = (1.0 - sponge) * f_post + sponge * feq0;
                    }
                    h->f_next[dst * Q + q] = f_post;
                }
            }
    double* t = h->f_curr;
    h->f_curr = h->f_next;
    h->f_next = t;
}

/* Probe record (06:1085-1092) */
void orc_record_probes(orc_handle* h)
{
    if (h->nprobe == 0) return;
    if (h->steps_rec == h->steps_cap)
    {
        h->steps_cap = h->steps_cap ? 2 * h->steps_cap : 1024;
        h->series = (double*)realloc(h->series, (size_t)h->steps_cap * h->nprobe * sizeof(double));
    }
    double* row = h->series + (size_t)h->steps_rec * h->nprobe;
    for (int p = 0; p < h->nprobe; ++p)
        row[p] = h->probe_idx[p] >= 0 ? h->rho[h->probe_idx[p]] - 1.0 : NAN;
    h->steps_rec++;
}

/* The body of LBMSolver::run (06:1077-1092) for steps s .. s+n-1. */
void orc_step(orc_handle* h, int nsteps)
{
    for (int n = 0; n < nsteps; ++n)
    {
        if (h->cfg.scheme == LBM_SCHEME_A)
        {
            step_a(h, h->step);   /* the field source acts inside the step */
        }
        else
        {
            const double t = h->step * h->dt;
            orc_apply_source(h, t);
            orc_exchange_halos(h);
            orc_step_collision_bgk(h);
        }
        orc_record_probes(h);
        h->step++;
    }
}

/* ---------------------------------------------------------------- access */

void orc_get_dims(orc_handle* h, int* n3, int* n3_halo)
{
    if (n3) { n3[0] = h->NXg; n3[1] = h->NYg; n3[2] = h->NZg; }
    if (n3_halo) { n3_halo[0] = h->nx_t; n3_halo[1] = h->ny_t; n3_halo[2] = h->nz_t; }
}
double orc_get_dt(orc_handle* h) { return h->dt; }
void orc_get_f(orc_handle* h, double* out) { memcpy(out, h->f_curr, h->Nloc * Q * sizeof(double)); }
void orc_set_f(orc_handle* h, const double* in) { memcpy(h->f_curr, in, h->Nloc * Q * sizeof(double)); }
/* Scheme A initial state at rest with density 1 + rho' at interior fluid
 * cells (01:183-205); rho_prime: nx*ny*nz values, x fastest. */
void orc_set_density(orc_handle* h, const double* rho_prime)
{
    const lbm_config* c = &h->cfg;
    for (int k = 1; k <= h->nz; ++k)
        for (int j = 1; j <= h->ny; ++j)
            for (int i = 1; i <= h->nx; ++i)
            {
                const size_t idx = loc(h, i, j, k);
                if (h->mask[idx] == SOLID) continue;
                const double r = 1.0 + rho_prime[((size_t)(k - 1) * h->ny + (j - 1)) * h->nx + (i - 1)];
                h->rho[idx] = r;
                for (int q = 0; q < Q; ++q) h->f_curr[idx * Q + q] = feq_a(q, r, c->flow[0], c->flow[1], c->flow[2]);
            }
}
void orc_get_mask(orc_handle* h, unsigned char* out) { memcpy(out, h->mask, h->Nloc); }
void orc_get_rho(orc_handle* h, double* out) { memcpy(out, h->rho, h->Nloc * sizeof(double)); }
void orc_get_sponge(orc_handle* h, double* out) { memcpy(out, h->sponge, h->Nloc * sizeof(double)); }
void orc_get_tau_a(orc_handle* h, double* out)
{
    for (size_t i = 0; i < h->Nloc; ++i) out[i] = h->tau_a ? h->tau_a[i] : h->cfg.tau;
}
void orc_get_ground_height(orc_handle* h, double* out)
{
    memcpy(out, h->gH, (size_t)h->nx_t * h->ny_t * sizeof(double));
}
long orc_get_probes(orc_handle* h, double* out, long capacity)
{
    long n = h->steps_rec * h->nprobe;
    if (n > capacity) return -1;
    if (n) memcpy(out, h->series, (size_t)n * sizeof(double));
    return h->steps_rec;
}

/* ---------------------------------------------------------------- adjoint (FP64)
 *
 * Discrete adjoint of orc_step for the misfit
 *     L = 1/2 sum_s sum_p (probe_s[p] - observed[s][p])^2,
 * the checker of the GPU adjoint.  The reference has no adjoint; this is
 * derived here from the forward restatement above and shares no code with
 * the GPU version: the transposed pull is a scatter, the BGK and ghost
 * Jacobians are differentiated in (rho, u) variables in full-population form,
 * and one checkpoint level (every K steps) is recomputed with all its states
 * stored.  Per step s, going backwards, with lamG = dL/d(post-collision
 * populations of step s):
 *   lamF  = J_bgk(F)^T lamG (+ residual at the probe cells, every q)
 *   lamHt = pull^T lamF                                 (halo included)
 *   lamH  = lamHt(interior) + J_ghost^T lamHt(open-face halo)
 *   dL/dmass_s = sum_c w_hat_c sum_q W_q lamH[c][q]; lamG(s-1) = lamH.
 */

/* Normalised injection weights of source s at its current position and their
 * derivatives with respect to the position; returns the cell count. */
static int adj_source_cells(const orc_handle* h, const src_t* s, size_t* idx, double* wh, double* dwh)
{
    const lbm_config* c = &h->cfg;
    const double DX = c->dx;
    double w[125], dw[375];
    int n = 0;
    if (s->s.injection == LBM_INJECT_TRILINEAR)
    {
        const double fx = (s->cx - c->x_min) / DX - 0.5, fy = (s->cy - c->y_min) / DX - 0.5,
                     fz = (s->cz - c->z_min) / DX - 0.5;
        const int i0 = (int)floor(fx), j0 = (int)floor(fy), k0 = (int)floor(fz);
        const double t[3] = {fx - i0, fy - j0, fz - k0};
        for (int b = 0; b < 8; ++b)
        {
            const int o[3] = {b & 1, (b >> 1) & 1, b >> 2};
            const int gi = i0 + o[0], gj = j0 + o[1], gk = k0 + o[2];
            if (!cell_in_grid(h, gi, gj, gk)) continue;
            const size_t id = loc(h, gi + 1, gj + 1, gk + 1);
            if (h->mask[id] != FLUID) continue;
            double f1[3], d1[3];
            for (int a = 0; a < 3; ++a)
            {
                f1[a] = o[a] ? t[a] : 1.0 - t[a];
                d1[a] = (o[a] ? 1.0 : -1.0) / DX;
            }
            idx[n] = id;
            w[n] = f1[0] * f1[1] * f1[2];
            dw[3 * n] = d1[0] * f1[1] * f1[2];
            dw[3 * n + 1] = f1[0] * d1[1] * f1[2];
            dw[3 * n + 2] = f1[0] * f1[1] * d1[2];
            ++n;
        }
    }
    else
    {
        const int R = s->s.radius;
        const double sig2 = (s->s.sigma_cells * DX) * (s->s.sigma_cells * DX);
        const int ic = (int)floor((s->cx - c->x_min) / DX), jc = (int)floor((s->cy - c->y_min) / DX),
                  kc = (int)floor((s->cz - c->z_min) / DX);
        if (ic < -R || ic >= h->NXg + R || jc < -R || jc >= h->NYg + R || kc < -R || kc >= h->NZg + R) return 0;
        for (int gk = kc - R; gk <= kc + R; ++gk)
            for (int gj = jc - R; gj <= jc + R; ++gj)
                for (int gi = ic - R; gi <= ic + R; ++gi)
                {
                    if (!cell_in_grid(h, gi, gj, gk)) continue;
                    const size_t id = loc(h, gi + 1, gj + 1, gk + 1);
                    if (h->mask[id] != FLUID) continue;
                    const double d[3] = {c->x_min + (gi + 0.5) * DX - s->cx, c->y_min + (gj + 0.5) * DX - s->cy,
                                         c->z_min + (gk + 0.5) * DX - s->cz};
                    idx[n] = id;
                    w[n] = exp(-0.5 * (d[0] * d[0] + d[1] * d[1] + d[2] * d[2]) / sig2);
                    for (int a = 0; a < 3; ++a) dw[3 * n + a] = w[n] * d[a] / sig2;
                    ++n;
                }
    }
    double S = 0.0, dS[3] = {0.0, 0.0, 0.0};
    for (int m = 0; m < n; ++m)
    {
        S += w[m];
        for (int a = 0; a < 3; ++a) dS[a] += dw[3 * m + a];
    }
    if (S < 1e-30) return 0;
    for (int m = 0; m < n; ++m)
    {
        wh[m] = w[m] / S;
        for (int a = 0; a < 3; ++a) dwh[3 * m + a] = dw[3 * m + a] / S - w[m] * dS[a] / (S * S);
    }
    return n;
}

/* macroscopic state of populations g: r = sum g, u = sum c g / r */
static void adj_macro(const double* g, double* r, double* u)
{
    double s = 0.0, m[3] = {0.0, 0.0, 0.0};
    for (int q = 0; q < Q; ++q)
    {
        s += g[q];
        m[0] += g[q] * EX[q];
        m[1] += g[q] * EY[q];
        m[2] += g[q] * EZ[q];
    }
    *r = s;
    for (int a = 0; a < 3; ++a) u[a] = m[a] / s;
}

/* For weights lam: a = sum_q lam_q feq_q(r,u) / r and
 * b_a = sum_q lam_q W_q r (3 c_qa + 9 (c_q.u) c_qa - 3 u_a), so that
 * sum_q lam_q d feq_q / d g_p = a d r/d g_p + b . d u / d g_p. */
static void adj_feq_weights(const double* lam, double r, const double* u, double* a, double* b)
{
    *a = 0.0;
    b[0] = b[1] = b[2] = 0.0;
    for (int q = 0; q < Q; ++q)
    {
        const double cq[3] = {EX[q], EY[q], EZ[q]};
        const double cu = cq[0] * u[0] + cq[1] * u[1] + cq[2] * u[2];
        *a += lam[q] * feq(q, r, u[0], u[1], u[2]) / r;
        for (int k = 0; k < 3; ++k) b[k] += lam[q] * W[q] * r * (3.0 * cq[k] + 9.0 * cu * cq[k] - 3.0 * u[k]);
    }
}

/* lamF = J_bgk(F)^T lamG at one FLUID cell (sponge s, omega om). */
static void adj_bgk(const double* F, const double* lamG, double om, double s, double* lamF)
{
    double r, u[3], a, b[3];
    adj_macro(F, &r, u);
    adj_feq_weights(lamG, r, u, &a, b);
    const double keep = s > 1e-12 ? 1.0 - s : 1.0;
    for (int p = 0; p < Q; ++p)
    {
        const double cp[3] = {EX[p], EY[p], EZ[p]};
        double t = a;
        for (int k = 0; k < 3; ++k) t += b[k] * (cp[k] - u[k]) / r;
        lamF[p] = keep * ((1.0 - om) * lamG[p] + om * t);
    }
}

/* Adds J_ghost^T lamB to lamI for the open-boundary ghost built from
 * interior populations gI (nscbc_ghost). */
static void adj_ghost(const double* gI, const double* lamB, int axis, int side, double* lamI)
{
    double rI, u[3];
    adj_macro(gI, &rI, u);
    const double pI = CS2 * (rI - 1.0);
    const double W_ = side == 0 ? u[axis] - pI / CS : u[axis] + pI / CS;
    const double pB = side == 0 ? -0.5 * CS * W_ : 0.5 * CS * W_;
    const double rhoB = 1.0 + pB / CS2;
    double uB[3] = {u[0], u[1], u[2]};
    uB[axis] = 0.5 * W_;
    double aB, bB[3], aI, bI[3];
    adj_feq_weights(lamB, rhoB, uB, &aB, bB);
    adj_feq_weights(lamB, rI, u, &aI, bI);
    for (int p = 0; p < Q; ++p)
    {
        const double cp[3] = {EX[p], EY[p], EZ[p]};
        double du[3];
        for (int k = 0; k < 3; ++k) du[k] = (cp[k] - u[k]) / rI;   /* d u_k / d g_p */
        const double dW = du[axis] + (side == 0 ? -CS : CS);       /* dp_I/dg_p = CS2, / CS */
        const double drhoB = (side == 0 ? -0.5 : 0.5) * CS * dW / CS2;
        double duB[3] = {du[0], du[1], du[2]};
        duB[axis] = 0.5 * dW;
        double t = lamB[p] + aB * drhoB - aI;
        for (int k = 0; k < 3; ++k) t += bB[k] * duB[k] - bI[k] * du[k];
        lamI[p] += t;
    }
}

int orc_adjoint_grad(orc_handle* h, int nsteps, const double* observed, int K, double* loss, double* grad_pos,
                     double* grad_signal, double* predicted)
{
    if (h->nsrc != 1 || h->nprobe < 1 || nsteps < 1 || h->step != 0) return LBM_ERR_STATE;
    if (K < 1) K = (int)ceil(sqrt((double)nsteps));
    if (K > nsteps) K = nsteps;
    const int T = nsteps, NC = (T + K - 1) / K, np = h->nprobe;
    const int nx = h->nx, ny = h->ny, nz = h->nz;
    const size_t NF = h->Nloc * Q;
    const double om = 1.0 / h->cfg.tau;
    const lbm_config* c = &h->cfg;
    src_t* S = &h->srcs[0];
    double* rest = (double*)malloc(NF * sizeof(double));
    double* ck = (double*)malloc((size_t)NC * NF * sizeof(double));
    double* store = (double*)malloc((size_t)K * NF * sizeof(double));
    double* lamG = (double*)calloc(NF, sizeof(double));
    double* lamF = (double*)calloc(NF, sizeof(double));
    double* lamH = (double*)calloc(NF, sizeof(double));
    double* pred = (double*)malloc((size_t)T * np * sizeof(double));
    double* res = (double*)calloc((size_t)T * np, sizeof(double));
    double* mass = (double*)malloc((size_t)T * sizeof(double));
    if (!rest || !ck || !store || !lamG || !lamF || !lamH || !pred || !res || !mass)
    {
        free(rest); free(ck); free(store); free(lamG); free(lamF); free(lamH); free(pred); free(res); free(mass);
        return LBM_ERR_OUT_OF_MEMORY;
    }
    memcpy(rest, h->f_curr, NF * sizeof(double));

    /* forward: checkpoints before the source of steps 0, K, 2K, ... */
    for (int s = 0; s < T; ++s)
    {
        if (s % K == 0) memcpy(ck + (size_t)(s / K) * NF, h->f_curr, NF * sizeof(double));
        const double t = s * h->dt;
        mass[s] = source_value(h, S, t) * h->dt * S->s.gain;
        orc_apply_source(h, t);
        orc_exchange_halos(h);
        orc_step_collision_bgk(h);
        for (int p = 0; p < np; ++p)
            pred[(size_t)s * np + p] = h->probe_idx[p] >= 0 ? h->rho[h->probe_idx[p]] - 1.0 : NAN;
    }
    double Ls = 0.0;
    for (int s = 0; s < T; ++s)
        for (int p = 0; p < np; ++p)
        {
            const size_t n = (size_t)s * np + p;
            if (h->probe_idx[p] < 0 || isnan(observed[n])) continue;
            const double r = pred[n] - observed[n];
            Ls += 0.5 * r * r;
            if (h->mask[h->probe_idx[p]] == FLUID) res[n] = r;
        }

    /* backward, one checkpoint segment at a time */
    size_t cidx[125];
    double wh[125], dwh[375];
    double gp[3] = {0.0, 0.0, 0.0};
    for (int g = NC - 1; g >= 0; --g)
    {
        const int a0 = g * K, a1 = (a0 + K < T) ? a0 + K : T;
        memcpy(h->f_curr, ck + (size_t)g * NF, NF * sizeof(double));
        for (int s = a0; s < a1; ++s)
        {
            orc_apply_source(h, s * h->dt);
            orc_exchange_halos(h);
            memcpy(store + (size_t)(s - a0) * NF, h->f_curr, NF * sizeof(double));
            if (s + 1 < a1) orc_step_collision_bgk(h);
        }
        for (int s = a1 - 1; s >= a0; --s)
        {
            const double* Ht = store + (size_t)(s - a0) * NF;
            /* lamF = J_bgk^T lamG; SOLID cells pass through */
            #pragma omp parallel for collapse(2)
            for (int k = 1; k <= nz; ++k)
                for (int j = 1; j <= ny; ++j)
                    for (int i = 1; i <= nx; ++i)
                    {
                        const size_t y = loc(h, i, j, k);
                        if (h->mask[y] == SOLID)
                        {
                            for (int q = 0; q < Q; ++q) lamF[y * Q + q] = lamG[y * Q + q];
                            continue;
                        }
                        double F[Q];
                        for (int q = 0; q < Q; ++q)
                        {
                            const size_t src = loc(h, i - EX[q], j - EY[q], k - EZ[q]);
                            F[q] = h->mask[src] == SOLID ? Ht[y * Q + h->inv_q[q]] : Ht[src * Q + q];
                        }
                        adj_bgk(F, lamG + y * Q, om, h->sponge[y], lamF + y * Q);
                    }
            for (int p = 0; p < np; ++p)
                if (h->probe_idx[p] >= 0)
                    for (int q = 0; q < Q; ++q) lamF[(size_t)h->probe_idx[p] * Q + q] += res[(size_t)s * np + p];
            /* lamHt = pull^T lamF (scatter, serial: targets overlap) */
            memset(lamH, 0, NF * sizeof(double));
            for (int k = 1; k <= nz; ++k)
                for (int j = 1; j <= ny; ++j)
                    for (int i = 1; i <= nx; ++i)
                    {
                        const size_t y = loc(h, i, j, k);
                        for (int q = 0; q < Q; ++q)
                        {
                            const size_t src = loc(h, i - EX[q], j - EY[q], k - EZ[q]);
                            if (h->mask[src] == SOLID) lamH[y * Q + h->inv_q[q]] += lamF[y * Q + q];
                            else lamH[src * Q + q] += lamF[y * Q + q];
                        }
                    }
            /* ghosts of the open faces back onto their interior cells */
            for (int f = 0; f < 6; ++f)
            {
                if (c->face_bc[f] != LBM_BC_NSCBC) continue;
                const int axis = f / 2, side = f % 2;
                const int n0 = axis == 0 ? ny : nx, n1 = axis == 2 ? ny : nz;
                for (int v = 1; v <= n1; ++v)
                    for (int u = 1; u <= n0; ++u)
                    {
                        int I[3], G[3];
                        if (axis == 0) { I[1] = G[1] = u; I[2] = G[2] = v; }
                        else if (axis == 1) { I[0] = G[0] = u; I[2] = G[2] = v; }
                        else { I[0] = G[0] = u; I[1] = G[1] = v; }
                        const int nn[3] = {nx, ny, nz};
                        I[axis] = side ? nn[axis] : 1;
                        G[axis] = side ? nn[axis] + 1 : 0;
                        const size_t iI = loc(h, I[0], I[1], I[2]), iG = loc(h, G[0], G[1], G[2]);
                        adj_ghost(Ht + iI * Q, lamH + iG * Q, axis, side, lamH + iI * Q);
                    }
            }
            /* source: mu_s and nu_s; lamG of step s-1 = lamH on interior cells */
            drone_update(S, s * h->dt);
            const int n = adj_source_cells(h, S, cidx, wh, dwh);
            double mu = 0.0, nu[3] = {0.0, 0.0, 0.0};
            for (int m = 0; m < n; ++m)
            {
                double lw = 0.0;
                for (int q = 0; q < Q; ++q) lw += W[q] * lamH[cidx[m] * Q + q];
                mu += wh[m] * lw;
                for (int a = 0; a < 3; ++a) nu[a] += dwh[3 * m + a] * lw;
            }
            if (grad_signal) grad_signal[s] = mu * h->dt * S->s.gain;
            for (int a = 0; a < 3; ++a) gp[a] += mass[s] * nu[a];
            memset(lamG, 0, NF * sizeof(double));
            for (int k = 1; k <= nz; ++k)
                for (int j = 1; j <= ny; ++j)
                    for (int i = 1; i <= nx; ++i)
                    {
                        const size_t y = loc(h, i, j, k);
                        for (int q = 0; q < Q; ++q) lamG[y * Q + q] = lamH[y * Q + q];
                    }
        }
    }
    if (grad_pos) for (int a = 0; a < 3; ++a) grad_pos[a] = gp[a];
    if (predicted) memcpy(predicted, pred, (size_t)T * np * sizeof(double));
    *loss = Ls;
    memcpy(h->f_curr, rest, NF * sizeof(double));
    for (size_t i = 0; i < h->Nloc; ++i) h->rho[i] = 1.0;
    h->step = 0;
    free(rest); free(ck); free(store); free(lamG); free(lamF); free(lamH); free(pred); free(res); free(mass);
    return LBM_OK;
}
