/*
 * fss_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement, in plain C99 / FP64, of the reference's hot path for the
 * barotropic-vorticity right-hand side (cygnari/fast-sphere-sum, directory
 * Old-BVE-code/).  Only tests/, the smoke check and the CPU-baseline leg of
 * the benchmark load this file's library; the product never links it.
 *
 * Every function keeps the reference's operation order so that, compiled
 * with -ffp-contract=off on x86-64 against the same libm, it is bit-for-bit
 * identical to the reference headers built by oracle/Makefile (target
 * _ref/libref.so).  The LU arithmetic used by the reference's barycoords()
 * comes from Apple Accelerate, which is not available; the oracle pins it to
 * an unblocked, partial-pivot LU in LAPACK dgetf2/dgetrs order (the same
 * arithmetic as oracle/ref_shim/lapack_shim.c used to build the reference).
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* ---------------------------------------------------------------- vectors */

/* helpers.h:23-28 dot_prod: sequential sum starting from 0. */
static double dot3(const double *x, const double *y) {
    double sum = 0;
    sum += x[0] * y[0];
    sum += x[1] * y[1];
    sum += x[2] * y[2];
    return sum;
}

/* helpers.h:30-32 vec_norm */
static double norm3(const double *x) { return sqrt(dot3(x, x)); }

/* helpers.h:82-85 project_to_sphere: p[i] *= radius / norm */
static void project_to_sphere(double *p, double radius) {
    double n = norm3(p);
    for (int i = 0; i < 3; i++) p[i] *= radius / n;
}

/* helpers.h:87-92 project_to_sphere_2: radius * p[i] / norm */
static void project_to_sphere_2(const double *p, double radius, double *out) {
    double n = norm3(p);
    for (int i = 0; i < 3; i++) out[i] = radius * p[i] / n;
}

/* helpers.h:54-62 cross_product */
static void cross3(const double *x, const double *y, double *v) {
    v[0] = x[1] * y[2] - x[2] * y[1];
    v[1] = x[2] * y[0] - x[0] * y[2];
    v[2] = x[0] * y[1] - x[1] * y[0];
}

/* helpers.h:217-222 BVE_gfunc: cross * (1 / (1 - dot)) */
void orc_bve_gfunc(const double *x, const double *y, double *out) {
    double denom = 1 - dot3(x, y);
    cross3(x, y, out);
    double s = 1 / denom;
    for (int i = 0; i < 3; i++) out[i] *= s;
}

/* ------------------------------------------------------- triangle metrics */

/* helpers.h:179-181 circum_poly */
static double circum_poly(double a, double b, double c) { return a * a + b * b - c * c; }

/* helpers.h:165-177 tri_sides + helpers.h:183-196 tri_center */
void orc_tri_center(const double *p1, const double *p2, const double *p3, double radius,
                    double *cent) {
    double p23[3], p31[3], p12[3];
    for (int i = 0; i < 3; i++) {
        p23[i] = p2[i] - p3[i];
        p31[i] = p3[i] - p1[i];
        p12[i] = p1[i] - p2[i];
    }
    double a = norm3(p23), b = norm3(p31), c = norm3(p12);
    double scaling = (a + b + c) * (a + b - c) * (a - b + c) * (b + c - a);
    double coeff1 = a * a * circum_poly(b, c, a) / scaling;
    double coeff2 = b * b * circum_poly(c, a, b) / scaling;
    double coeff3 = c * c * circum_poly(a, b, c) / scaling;
    for (int k = 0; k < 3; k++) cent[k] = coeff1 * p1[k] + coeff2 * p2[k] + coeff3 * p3[k];
    project_to_sphere(cent, radius);
}

/* helpers.h:198-209 tri_radius: max chord from the centre (std::max order) */
double orc_tri_radius(const double *p1, const double *p2, const double *p3, const double *c) {
    double d1[3], d2[3], d3[3];
    for (int i = 0; i < 3; i++) {
        d1[i] = p1[i] - c[i];
        d2[i] = p2[i] - c[i];
        d3[i] = p3[i] - c[i];
    }
    double r1 = norm3(d1), r2 = norm3(d2), r3 = norm3(d3);
    double m = (r1 < r2) ? r2 : r1;
    return (m < r3) ? r3 : m;
}

/* helpers.h:94-115 sphere_tri_area (L'Huilier with chord-derived sides) */
double orc_sphere_tri_area(const double *p1, const double *p2, const double *p3, double radius) {
    double p1n[3], p2n[3], p3n[3];
    for (int i = 0; i < 3; i++) {
        p2n[i] = p2[i] - p3[i];
        p3n[i] = p3[i] - p1[i];
        p1n[i] = p1[i] - p2[i];
    }
    double a = acos(1 - 0.5 * dot3(p2n, p2n));
    double b = acos(1 - 0.5 * dot3(p3n, p3n));
    double c = acos(1 - 0.5 * dot3(p1n, p1n));
    double s = (a + b + c) / 2;
    double z = tan(s / 2) * tan((s - a) / 2) * tan((s - b) / 2) * tan((s - c) / 2);
    return 4 * radius * radius * atan(sqrt(z));
}

/* helpers.h:211-215 great_circ_dist */
double orc_great_circ_dist(const double *p1, const double *p2, double radius) {
    double s = dot3(p1, p2) / (norm3(p1) * norm3(p2));
    double lo = (s < -1.0) ? -1.0 : s;          /* std::max(s, -1.0) */
    double cl = (1.0 < lo) ? 1.0 : lo;          /* std::min(.., 1.0) */
    return acos(cl) * radius;
}

/* ------------------------------------------------------------ pinned LU */

/* 3x3 column-major LU with partial pivoting, LAPACK dgetf2 order: pivot is
 * the first row of maximal |a(i,k)|, rows swapped across all columns, the
 * column below the pivot scaled by the reciprocal, then the rank-1 update.
 * Solve in dgetrs order (row swaps, unit-lower forward, upper backward).
 * Mirrors the call dgesv_(3, 1, mat, 3, ipiv, coords, 3, info) made by
 * helpers.h:137-150 barycoords().  Returns the LAPACK info value. */
static int lu_solve3(double *a, double *b) {
    int ipiv[3];
    int info = 0;
    for (int k = 0; k < 3; k++) {
        int p = k;
        double mx = fabs(a[k + 3 * k]);
        for (int i = k + 1; i < 3; i++)
            if (fabs(a[i + 3 * k]) > mx) { mx = fabs(a[i + 3 * k]); p = i; }
        ipiv[k] = p;
        if (a[p + 3 * k] == 0.0) { if (!info) info = k + 1; continue; }
        if (p != k)
            for (int j = 0; j < 3; j++) {
                double t = a[k + 3 * j]; a[k + 3 * j] = a[p + 3 * j]; a[p + 3 * j] = t;
            }
        double r = 1.0 / a[k + 3 * k];
        for (int i = k + 1; i < 3; i++) a[i + 3 * k] *= r;
        for (int j = k + 1; j < 3; j++)
            for (int i = k + 1; i < 3; i++) a[i + 3 * j] -= a[i + 3 * k] * a[k + 3 * j];
    }
    if (info) return info;  /* dgesv returns before the solve */
    for (int k = 0; k < 3; k++) {
        int p = ipiv[k];
        if (p != k) { double t = b[k]; b[k] = b[p]; b[p] = t; }
    }
    for (int k = 0; k < 3; k++)
        for (int i = k + 1; i < 3; i++) b[i] -= a[i + 3 * k] * b[k];
    for (int k = 2; k >= 0; k--) {
        b[k] /= a[k + 3 * k];
        for (int i = 0; i < k; i++) b[i] -= a[i + 3 * k] * b[k];
    }
    return 0;
}

/* helpers.h:137-150 barycoords (unnormalised cone coordinates) */
void orc_barycoords(const double *p1, const double *p2, const double *p3, const double *p,
                    double *coords) {
    double mat[9] = {p1[0], p1[1], p1[2], p2[0], p2[1], p2[2], p3[0], p3[1], p3[2]};
    coords[0] = p[0]; coords[1] = p[1]; coords[2] = p[2];
    lu_solve3(mat, coords);
}

/* helpers.h:159-163 check_in_tri */
static int check_in_tri(const double *p1, const double *p2, const double *p3, const double *p) {
    double c[3];
    orc_barycoords(p1, p2, p3, p, c);
    return (c[0] >= 0) && (c[1] >= 0) && (c[2] >= 0);
}

/* ------------------------------------------------------ icosahedral tree */

/* Open-addressing hash of exact vertex coordinates; equality is the double
 * '==' of helpers.h:224-229 check_in_vec (so -0.0 and +0.0 hash alike). */
typedef struct { int64_t cap; int *slot; const double *verts; } vhash;

static uint64_t vkey(const double *v) {
    uint64_t h = 1469598103934665603ULL;
    for (int i = 0; i < 3; i++) {
        double x = (v[i] == 0.0) ? 0.0 : v[i];
        uint64_t b; memcpy(&b, &x, 8);
        h ^= b; h *= 1099511628211ULL; h ^= h >> 29;
    }
    return h;
}

static int vhash_find(vhash *h, const double *v, int insert_id) {
    uint64_t m = (uint64_t)h->cap - 1, i = vkey(v) & m;
    for (;;) {
        int id = h->slot[i];
        if (id < 0) {
            if (insert_id >= 0) h->slot[i] = insert_id;
            return -1;
        }
        const double *w = h->verts + 3 * (int64_t)id;
        if (w[0] == v[0] && w[1] == v[1] && w[2] == v[2]) return id;
        i = (i + 1) & m;
    }
}

/* Number of vertices after `levels` refinements and faces on levels 0..levels. */
void orc_icos_counts(int levels, int64_t *nverts, int64_t *nfaces_total) {
    int64_t p = 1, tot = 0;
    for (int l = 0; l <= levels; l++) { tot += 20 * p; if (l < levels) p *= 4; }
    *nverts = 10 * p + 2;
    *nfaces_total = tot;
}

/* icos_utils.h:15-133 icos_init.
 * verts[3*V]; tri_verts[3*F] and (optional) tri_info[4*F] with the levels
 * stored one after another (level l starts at face 20*(4^l-1)/3).  Vertex
 * dedupe uses a hash in place of the linear check_in_vec scan; the
 * first-insertion order is unchanged.  Returns the vertex count. */
int64_t orc_icos_init(int levels, double radius, double *verts, int *tri_verts, double *tri_info) {
    int64_t V, F;
    orc_icos_counts(levels, &V, &F);
    vhash h;
    h.cap = 1;
    while (h.cap < 2 * V + 16) h.cap <<= 1;
    h.slot = (int *)malloc(sizeof(int) * (size_t)h.cap);
    for (int64_t i = 0; i < h.cap; i++) h.slot[i] = -1;
    h.verts = verts;

    double phi = (1 + sqrt(5)) / 2;
    double base[12][3] = {{0, 1, phi}, {0, -1, phi}, {0, 1, -phi}, {0, -1, -phi},
                          {1, phi, 0}, {1, -phi, 0}, {-1, phi, 0}, {-1, -phi, 0},
                          {phi, 0, 1}, {phi, 0, -1}, {-phi, 0, 1}, {-phi, 0, -1}};
    int64_t nv = 0;
    for (int i = 0; i < 12; i++) {
        project_to_sphere_2(base[i], radius, verts + 3 * nv);
        vhash_find(&h, verts + 3 * nv, (int)nv);
        nv++;
    }
    static const int faces1[20][3] = {{1, 2, 9},  {1, 2, 11}, {1, 5, 7},  {1, 5, 9},   {1, 7, 11},
                                      {2, 6, 8},  {2, 6, 9},  {2, 8, 11}, {3, 4, 10},  {3, 4, 12},
                                      {3, 5, 7},  {3, 5, 10}, {3, 7, 12}, {4, 6, 8},   {4, 6, 10},
                                      {4, 8, 12}, {5, 9, 10}, {6, 9, 10}, {7, 11, 12}, {8, 11, 12}};
    for (int i = 0; i < 20; i++) {
        for (int j = 0; j < 3; j++) tri_verts[3 * i + j] = faces1[i][j] - 1;
        if (tri_info) {
            const double *v1 = verts + 3 * tri_verts[3 * i], *v2 = verts + 3 * tri_verts[3 * i + 1],
                         *v3 = verts + 3 * tri_verts[3 * i + 2];
            double *ti = tri_info + 4 * i;
            orc_tri_center(v1, v2, v3, radius, ti);
            ti[3] = orc_tri_radius(v1, v2, v3, ti);
        }
    }
    int64_t off = 0, nf = 20;
    for (int l = 0; l < levels; l++) {
        int64_t noff = off + nf;
        for (int64_t j = 0; j < nf; j++) {
            int iv1 = tri_verts[3 * (off + j)], iv2 = tri_verts[3 * (off + j) + 1],
                iv3 = tri_verts[3 * (off + j) + 2];
            double v1[3], v2[3], v3[3], v12[3], v23[3], v31[3];
            memcpy(v1, verts + 3 * (int64_t)iv1, 24);
            memcpy(v2, verts + 3 * (int64_t)iv2, 24);
            memcpy(v3, verts + 3 * (int64_t)iv3, 24);
            for (int k = 0; k < 3; k++) {
                v12[k] = v1[k] + v2[k];
                v23[k] = v2[k] + v3[k];
                v31[k] = v3[k] + v1[k];
            }
            for (int k = 0; k < 3; k++) { v12[k] *= 0.5; v23[k] *= 0.5; v31[k] *= 0.5; }
            project_to_sphere(v12, radius);
            project_to_sphere(v23, radius);
            project_to_sphere(v31, radius);
            int iv12 = vhash_find(&h, v12, -1);
            int iv13 = vhash_find(&h, v31, -1);
            int iv23 = vhash_find(&h, v23, -1);
            if (iv12 == -1) { iv12 = (int)nv; memcpy(verts + 3 * nv, v12, 24); vhash_find(&h, v12, iv12); nv++; }
            if (iv13 == -1) { iv13 = (int)nv; memcpy(verts + 3 * nv, v31, 24); vhash_find(&h, v31, iv13); nv++; }
            if (iv23 == -1) { iv23 = (int)nv; memcpy(verts + 3 * nv, v23, 24); vhash_find(&h, v23, iv23); nv++; }
            int *c = tri_verts + 3 * (noff + 4 * j);
            c[0] = iv1;  c[1] = iv13; c[2] = iv12;
            c[3] = iv3;  c[4] = iv23; c[5] = iv13;
            c[6] = iv2;  c[7] = iv12; c[8] = iv23;
            c[9] = iv12; c[10] = iv13; c[11] = iv23;
            if (tri_info) {
                double *ti = tri_info + 4 * (noff + 4 * j);
                orc_tri_center(v1, v12, v31, radius, ti);
                ti[3] = orc_tri_radius(v1, v12, v31, ti);
                orc_tri_center(v3, v23, v31, radius, ti + 4);
                ti[7] = orc_tri_radius(v3, v23, v31, ti + 4);
                orc_tri_center(v2, v12, v23, radius, ti + 8);
                ti[11] = orc_tri_radius(v2, v12, v23, ti + 8);
                orc_tri_center(v12, v31, v23, radius, ti + 12);
                ti[15] = orc_tri_radius(v12, v31, v23, ti + 12);
            }
        }
        off = noff;
        nf *= 4;
    }
    free(h.slot);
    return nv;
}

/* helpers.h:344-360 area_init: A_i += area/3 over the faces in order. */
void orc_area_init(int64_t n, const double *state5, int64_t ntri, const int *tris, double *area) {
    for (int64_t i = 0; i < n; i++) area[i] = 0;
    for (int64_t t = 0; t < ntri; t++) {
        int i1 = tris[3 * t], i2 = tris[3 * t + 1], i3 = tris[3 * t + 2];
        double a = orc_sphere_tri_area(state5 + 5 * (int64_t)i1, state5 + 5 * (int64_t)i2,
                                       state5 + 5 * (int64_t)i3, 1);
        area[i1] += a / 3.0;
        area[i2] += a / 3.0;
        area[i3] += a / 3.0;
    }
}

/* helpers.h:117-124 lat_lon */
static void lat_lon(const double *p, double *lat, double *lon) {
    double x = p[0], y = p[1], z = p[2];
    *lat = M_PI / 2 - atan2(sqrt(x * x + y * y), z);
    *lon = atan2(y, x);
}

/* vorticity_functions.h:13-24 rossby_haurwitz_4 (reference constants). */
void orc_rossby_haurwitz_4(int64_t n, double *state5) {
    for (int64_t i = 0; i < n; i++) {
        double lat, lon;
        lat_lon(state5 + 5 * i, &lat, &lon);
        state5[5 * i + 4] = 2 + lat;
        state5[5 * i + 3] = 2 * M_PI * sin(lat) / 7.0 + 30.0 * sin(lat) * pow(cos(lat), 4) * cos(4 * lon);
    }
}

/* ------------------------------------------- seeded RH wave + Gaussian vortices
 *
 * The benchmark's input field, restated from its definition (no reference
 * counterpart: the reference hard-codes the RH constants and has one vortex):
 *
 *   zeta(x) = 2 w sin(lat) - K (R + 1)(R + 2) cos^R(lat) sin(lat) cos(R lon)
 *             + sum_v a_v exp(-(d(x, c_v) / width)^2),   R = 4, w = K = amp,
 *
 * d the great-circle distance; vortex centres uniform on the sphere (z and
 * longitude uniform), amplitudes normal with variance 2 pi^2; the
 * area-weighted mean is removed; tracer = 2 + lat.  Random numbers: the
 * 64-bit Mersenne twister MT19937-64 (Matsumoto and Nishimura, 2000; the
 * generator C++ names std::mt19937_64), uniform doubles from its top 53
 * bits, normals by the Box-Muller transform.  Per vortex the draws are
 * z, lon, u1, u2 in that order. */

typedef struct {
    uint64_t mt[312];
    int i;
} mt64;

static void mt64_seed(mt64 *g, uint64_t seed) {
    g->mt[0] = seed;
    for (int i = 1; i < 312; i++) g->mt[i] = 6364136223846793005ULL * (g->mt[i - 1] ^ (g->mt[i - 1] >> 62)) + (uint64_t)i;
    g->i = 312;
}

static uint64_t mt64_next(mt64 *g) {
    const uint64_t upper = 0xFFFFFFFF80000000ULL, lower = 0x7FFFFFFFULL, a = 0xB5026F5AA96619E9ULL;
    if (g->i >= 312) {
        for (int k = 0; k < 312; k++) {
            const uint64_t x = (g->mt[k] & upper) | (g->mt[(k + 1) % 312] & lower);
            g->mt[k] = g->mt[(k + 156) % 312] ^ (x >> 1) ^ ((x & 1ULL) ? a : 0ULL);
        }
        g->i = 0;
    }
    uint64_t x = g->mt[g->i++];
    x ^= (x >> 29) & 0x5555555555555555ULL;
    x ^= (x << 17) & 0x71D67FFFEDA60000ULL;
    x ^= (x << 37) & 0xFFF7EEE000000000ULL;
    x ^= x >> 43;
    return x;
}

static double mt64_uniform(mt64 *g) { return (double)(mt64_next(g) >> 11) * (1.0 / 9007199254740992.0); }

/* Raw generator output, for pinning the generator itself. */
void orc_mt64_draws(uint64_t seed, int64_t count, uint64_t *out) {
    mt64 g;
    mt64_seed(&g, seed);
    for (int64_t k = 0; k < count; k++) out[k] = mt64_next(&g);
}

void orc_rh_vortices(int64_t n, double *state5, const double *area, double amp, int nvort, double width,
                     uint64_t seed) {
    mt64 g;
    mt64_seed(&g, seed);
    double *cen = (double *)malloc(sizeof(double) * 4 * (size_t)(nvort > 0 ? nvort : 1));
    for (int v = 0; v < nvort; v++) {
        const double z = 2 * mt64_uniform(&g) - 1;
        const double lon = 2 * M_PI * mt64_uniform(&g);
        const double rho = sqrt(fmax(0.0, 1 - z * z));
        const double u1 = 1.0 - mt64_uniform(&g), u2 = mt64_uniform(&g);
        cen[4 * v + 0] = rho * cos(lon);
        cen[4 * v + 1] = rho * sin(lon);
        cen[4 * v + 2] = z;
        cen[4 * v + 3] = sqrt(2 * M_PI * M_PI) * sqrt(-2 * log(u1)) * cos(2 * M_PI * u2);
    }
    const double w = amp, K = amp;
    double num = 0, den = 0;
    for (int64_t i = 0; i < n; i++) {
        double *p = state5 + 5 * i;
        double lat, lon;
        lat_lon(p, &lat, &lon);
        double zeta = 2 * w * sin(lat) - K * (4 + 1) * (4 + 2) * pow(cos(lat), 4) * sin(lat) * cos(4 * lon);
        for (int v = 0; v < nvort; v++) {
            const double *c = cen + 4 * v;
            const double cosd = fmin(1.0, fmax(-1.0, p[0] * c[0] + p[1] * c[1] + p[2] * c[2]));
            const double d = acos(cosd) / width;
            zeta += c[3] * exp(-(d * d));
        }
        p[3] = zeta;
        p[4] = 2 + lat;
        if (area) {
            num += zeta * area[i];
            den += area[i];
        }
    }
    if (area && den > 0)
        for (int64_t i = 0; i < n; i++) state5[5 * i + 3] -= num / den;
    free(cen);
}

/* ------------------------------------------------------------ direct sum */

/* rhs_eval.h:15-32 rhs_direct_sum, one target row (sequential j order). */
static void direct_row(int64_t i, int64_t n, const double *s, const double *area, double *pc) {
    const double *xi = s + 5 * i;
    pc[0] = 0; pc[1] = 0; pc[2] = 0;
    for (int64_t j = 0; j < n; j++) {
        if (i == j) continue;
        double g[3];
        orc_bve_gfunc(xi, s + 5 * j, g);
        double w = s[5 * j + 3] * area[j];
        for (int k = 0; k < 3; k++) g[k] *= w;
        for (int k = 0; k < 3; k++) pc[k] += g[k];
    }
}

typedef struct {
    int64_t n, lo, hi;
    const double *s, *area;
    const int64_t *rows;
    double omega, *out;
    int mode; /* 0: full rhs_func rows into out5 ; 1: sampled rows into out3 */
} drow_job;

static void *drow_worker(void *p) {
    drow_job *J = (drow_job *)p;
    const double scale = -1.0 / (4.0 * M_PI);
    for (int64_t r = J->lo; r < J->hi; r++) {
        int64_t i = J->rows ? J->rows[r] : r;
        double pc[3];
        direct_row(i, J->n, J->s, J->area, pc);
        if (J->mode == 0) {
            double *m = J->out + 5 * i;
            /* rhs_func: zero, sum, scale all 5 entries, then dzeta/dt. */
            m[0] = pc[0] * scale; m[1] = pc[1] * scale; m[2] = pc[2] * scale;
            m[3] = 0.0 * scale;   m[4] = 0.0 * scale;
            m[3] = -2 * J->omega * m[2];
        } else {
            double *m = J->out + 3 * r;
            m[0] = pc[0] * scale; m[1] = pc[1] * scale; m[2] = pc[2] * scale;
        }
    }
    return NULL;
}

static void run_rows(drow_job base, int64_t nrows, int threads) {
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    pthread_t th[256];
    drow_job jobs[256];
    for (int t = 0; t < threads; t++) {
        jobs[t] = base;
        jobs[t].lo = nrows * t / threads;
        jobs[t].hi = nrows * (t + 1) / threads;
        if (threads == 1) { drow_worker(&jobs[t]); return; }
        pthread_create(&th[t], NULL, drow_worker, &jobs[t]);
    }
    for (int t = 0; t < threads; t++) pthread_join(th[t], NULL);
}

/* rhs_eval.h:47-56 rhs_func with use_fast == false.  Rows are independent,
 * so splitting them over threads keeps every value bit-identical. */
void orc_rhs_direct(int64_t n, const double *state5, const double *area, double omega,
                    double *modify5, int threads) {
    drow_job b = {n, 0, 0, state5, area, NULL, omega, modify5, 0};
    run_rows(b, n, threads);
}

/* Velocity (already scaled by -1/4pi) at a subset of target rows. */
void orc_rhs_direct_rows(int64_t n, const double *state5, const double *area, int64_t nrows,
                         const int64_t *rows, double *out3, int threads) {
    drow_job b = {n, 0, 0, state5, area, rows, 0.0, out3, 1};
    run_rows(b, nrows, threads);
}

/* Stream function psi_i = -(1/4pi) sum_{j!=i} zeta_j A_j log(1 - x_i.x_j).
 * No counterpart exists in the reference; this is the formula itself. */
void orc_stream_rows(int64_t n, const double *state5, const double *area, int64_t nrows,
                     const int64_t *rows, double *psi) {
    for (int64_t r = 0; r < nrows; r++) {
        int64_t i = rows ? rows[r] : r;
        double acc = 0;
        for (int64_t j = 0; j < n; j++) {
            if (j == i) continue;
            acc += state5[5 * j + 3] * area[j] * log(1 - dot3(state5 + 5 * i, state5 + 5 * j));
        }
        psi[r] = acc * (-1.0 / (4.0 * M_PI));
    }
}

/* ------------------------------------------------------------------- RK4 */

/* helpers.h:362-372 project_points */
void orc_project_points(int64_t n, double *s, double omega) {
    for (int64_t i = 0; i < n; i++) {
        double p[3] = {s[5 * i], s[5 * i + 1], s[5 * i + 2]};
        project_to_sphere(p, 1.0);
        double dz = p[2] - s[5 * i + 2];
        s[5 * i] = p[0]; s[5 * i + 1] = p[1]; s[5 * i + 2] = p[2];
        s[5 * i + 3] += -2 * omega * dz;
    }
}

/* One RK4 step in the order of new_dynamics.cpp:281-340 (the intended
 * loop: stage states s + c*dt*k, each projected; k1 + 2k2 + 2k3 + k4 scaled
 * by dt/6, added, projected).  Uses the FP64 direct sum as the RHS. */
void orc_rk4_step(int64_t n, double *state5, const double *area, double omega, double dt,
                  int threads) {
    size_t sz = sizeof(double) * 5 * (size_t)n;
    double *k1 = malloc(sz), *k2 = malloc(sz), *k3 = malloc(sz), *k4 = malloc(sz), *t = malloc(sz);
    orc_rhs_direct(n, state5, area, omega, k1, threads);
    for (int64_t i = 0; i < 5 * n; i++) { t[i] = k1[i] * (dt / 2); t[i] += state5[i]; }
    orc_project_points(n, t, omega);
    orc_rhs_direct(n, t, area, omega, k2, threads);
    for (int64_t i = 0; i < 5 * n; i++) { t[i] = k2[i] * (dt / 2); t[i] += state5[i]; }
    orc_project_points(n, t, omega);
    orc_rhs_direct(n, t, area, omega, k3, threads);
    for (int64_t i = 0; i < 5 * n; i++) { t[i] = k3[i] * dt; t[i] += state5[i]; }
    orc_project_points(n, t, omega);
    orc_rhs_direct(n, t, area, omega, k4, threads);
    for (int64_t i = 0; i < 5 * n; i++) {
        double c = k1[i];
        c += k2[i] * 2;
        c += k3[i] * 2;
        c += k4[i];
        c *= dt / 6;
        state5[i] += c;
    }
    orc_project_points(n, state5, omega);
    free(k1); free(k2); free(k3); free(k4); free(t);
}

/* ------------------------------------------------- tree membership, MAC */

/* icos_utils.h:145-190 point_assign / points_assign for a fresh tree:
 * loc[l*n + i] is the face of particle i on level l, or -1 when no face
 * passed check_in_tri (the reference then searches children of face 0 on
 * the next level, because its tree_point_locs entry stays 0). */
void orc_points_assign(int tree_levels, const double *verts, const int *tri_verts, int64_t n,
                       const double *state5, int *loc) {
    for (int64_t i = 0; i < n; i++) {
        const double *p = state5 + 5 * i;
        int prev = 0;
        int64_t off = 0, nf = 20;
        for (int l = 0; l < tree_levels; l++) {
            int lb = (l > 0) ? 4 * prev : 0, ub = (l > 0) ? lb + 4 : 20;
            int found = -1;
            for (int j = lb; j < ub; j++) {
                const int *tv = tri_verts + 3 * (off + j);
                if (check_in_tri(verts + 3 * (int64_t)tv[0], verts + 3 * (int64_t)tv[1],
                                 verts + 3 * (int64_t)tv[2], p)) { found = j; break; }
            }
            loc[(int64_t)l * n + i] = found;
            prev = (found >= 0) ? found : 0;
            off += nf;
            nf *= 4;
        }
    }
}

/* fast_rhs.h:16-91 tree_traverse with a FIFO queue.
 * counts: per-face particle counts, levels concatenated.  tri_info: as from
 * orc_icos_init.  Output records of 7 ints (lev_t, lev_s, t, s, n_t, n_s,
 * type) with type 0 "pp", 1 "pc", 2 "cp", 3 "cc" (first letter: target).
 * Returns the number of records, or -(needed) if out_cap is too small. */
int64_t orc_tree_traverse(int tree_levels, double theta, int many_count, const int *counts,
                          const double *tri_info, double radius, int *out, int64_t out_cap) {
    int64_t lev_off[32];
    int64_t o = 0, nf = 20;
    for (int l = 0; l < 32; l++) { lev_off[l] = o; o += nf; if (l < 31 && nf < ((int64_t)1 << 40)) nf *= 4; }
    int64_t qcap = 1 << 16, qh = 0, qt = 0, nout = 0;
    int *q = (int *)malloc(sizeof(int) * 4 * (size_t)qcap);
#define QPUSH(a, b, c, d)                                                                   \
    do {                                                                                    \
        if (qt - qh == qcap) {                                                              \
            int *nq = (int *)malloc(sizeof(int) * 8 * (size_t)qcap);                        \
            for (int64_t z = 0; z < qcap; z++)                                              \
                memcpy(nq + 4 * z, q + 4 * ((qh + z) % qcap), 16);                          \
            free(q); q = nq; qh = 0; qt = qcap; qcap *= 2;                                  \
        }                                                                                   \
        int *e_ = q + 4 * (qt % qcap);                                                      \
        e_[0] = (a); e_[1] = (b); e_[2] = (c); e_[3] = (d);                                 \
        qt++;                                                                               \
    } while (0)
    for (int i = 0; i < 20; i++)
        for (int j = 0; j < 20; j++) QPUSH(i, j, 0, 0);
    while (qt > qh) {
        int *e = q + 4 * (qh % qcap);
        int ct = e[0], cs = e[1], lt = e[2], ls = e[3];
        qh++;
        int nt = counts[lev_off[lt] + ct], ns = counts[lev_off[ls] + cs];
        if (nt == 0 || ns == 0) continue;
        const double *ti = tri_info + 4 * (lev_off[lt] + ct), *si = tri_info + 4 * (lev_off[ls] + cs);
        double dist = orc_great_circ_dist(ti, si, radius);
        double sep = (ti[3] + si[3]) / dist;
        int rec = -1;
        if (dist > 0 && sep < theta) {
            rec = ((nt > many_count) ? 2 : 0) + ((ns > many_count) ? 1 : 0);
        } else if (nt < many_count && ns < many_count) {
            rec = 0;
        } else if (lt == tree_levels - 1 && ls == tree_levels - 1) {
            rec = 0;
        } else if (lt == tree_levels - 1) {
            for (int c = 0; c < 4; c++) QPUSH(ct, 4 * cs + c, lt, ls + 1);
        } else if (ls == tree_levels - 1) {
            for (int c = 0; c < 4; c++) QPUSH(4 * ct + c, cs, lt + 1, ls);
        } else if (nt >= ns) {
            for (int c = 0; c < 4; c++) QPUSH(4 * ct + c, cs, lt + 1, ls);
        } else {
            for (int c = 0; c < 4; c++) QPUSH(ct, 4 * cs + c, lt, ls + 1);
        }
        if (rec >= 0) {
            if (nout < out_cap) {
                int *r = out + 7 * nout;
                r[0] = lt; r[1] = ls; r[2] = ct; r[3] = cs; r[4] = nt; r[5] = ns; r[6] = rec;
            }
            nout++;
        }
    }
#undef QPUSH
    free(q);
    return (nout <= out_cap) ? nout : -nout;
}

/* ----------------------------------------------------------------- remesh */

/* helpers.h:152-157 norm_barycoords: cone coordinates scaled by the
 * reciprocal of their sum ((c0 + c1) + c2). */
static void norm_barycoords(const double *p1, const double *p2, const double *p3, const double *p,
                            double *c) {
    orc_barycoords(p1, p2, p3, p, c);
    const double r = 1.0 / (c[0] + c[1] + c[2]);
    for (int k = 0; k < 3; k++) c[k] *= r;
}

/* helpers.h:251-265 tri_interp: absolute vorticity zeta + 2 omega z and the
 * tracer, interpolated at the target with normalised barycentric
 * coordinates; zeta = interpolated - 2 omega z_target. */
static void tri_interp(const int *tv, const double *moved5, double *target5, int64_t i, double omega) {
    const double *v1 = moved5 + 5 * (int64_t)tv[0], *v2 = moved5 + 5 * (int64_t)tv[1],
                 *v3 = moved5 + 5 * (int64_t)tv[2];
    double *t = target5 + 5 * i;
    double b[3];
    norm_barycoords(v1, v2, v3, t, b);
    const double a1 = v1[3] + 2 * omega * v1[2];
    const double a2 = v2[3] + 2 * omega * v2[2];
    const double a3 = v3[3] + 2 * omega * v3[2];
    const double av = b[0] * a1 + b[1] * a2 + b[2] * a3;
    t[3] = av - 2 * omega * t[2];
    t[4] = b[0] * v1[4] + b[1] * v2[4] + b[2] * v3[4];
}

/* remesh.h:109-178 regrid_points2: every target point (its position kept)
 * takes the zeta and tracer interpolated from the first triangle of the
 * moved mesh that contains it, searched among the triangles adjacent to its
 * own vertex in increasing index order, then among all triangles in index
 * order.  The reference reads that adjacency from a CSV file it does not
 * contain; here it is built from `tris` in increasing index order.  Returns
 * the number of targets found in no triangle (left unchanged); *fallback
 * receives the number that needed the search over all triangles. */
/* Adjacency order: by corner key (keys[3 j + c] for corner c of triangle j),
 * or by triangle index when keys is NULL. */
static const uint64_t *g_sort_keys;
static int cmp_corner(const void *x, const void *y) {
    const int64_t a = *(const int64_t *)x, b = *(const int64_t *)y;
    const uint64_t ka = g_sort_keys ? g_sort_keys[a] : (uint64_t)a, kb = g_sort_keys ? g_sort_keys[b] : (uint64_t)b;
    return ka < kb ? -1 : (ka > kb ? 1 : 0);
}

int64_t orc_remesh_keyed(int64_t n, const double *moved5, double *target5, int64_t ntri, const int *tris,
                         const uint64_t *keys, double omega, int64_t *fallback) {
    int64_t *off = calloc((size_t)n + 1, sizeof(int64_t));
    int64_t *adj = malloc(sizeof(int64_t) * (size_t)(3 * ntri + 1));  /* corner ids 3 j + c */
    for (int64_t j = 0; j < 3 * ntri; j++) off[tris[j] + 1]++;
    for (int64_t i = 0; i < n; i++) off[i + 1] += off[i];
    int64_t *fill = malloc(sizeof(int64_t) * (size_t)(n + 1));
    memcpy(fill, off, sizeof(int64_t) * (size_t)(n + 1));
    for (int64_t j = 0; j < 3 * ntri; j++) adj[fill[tris[j]]++] = j;
    g_sort_keys = keys;
    for (int64_t i = 0; i < n; i++) qsort(adj + off[i], (size_t)(off[i + 1] - off[i]), sizeof(int64_t), cmp_corner);
    int64_t bad = 0, fb = 0;
    for (int64_t i = 0; i < n; i++) {
        const double *p = target5 + 5 * i;
        int64_t found = -1;
        for (int64_t a = off[i]; a < off[i + 1] && found < 0; a++) {
            const int *tv = tris + 3 * (adj[a] / 3);
            if (check_in_tri(moved5 + 5 * (int64_t)tv[0], moved5 + 5 * (int64_t)tv[1], moved5 + 5 * (int64_t)tv[2], p))
                found = adj[a] / 3;
        }
        if (found < 0) {
            fb++;
            for (int64_t j = 0; j < ntri && found < 0; j++) {
                const int *tv = tris + 3 * j;
                if (check_in_tri(moved5 + 5 * (int64_t)tv[0], moved5 + 5 * (int64_t)tv[1], moved5 + 5 * (int64_t)tv[2], p))
                    found = j;
            }
        }
        if (found < 0) { bad++; continue; }
        tri_interp(tris + 3 * found, moved5, target5, i, omega);
    }
    free(off); free(adj); free(fill);
    if (fallback) *fallback = fb;
    return bad;
}

int64_t orc_remesh(int64_t n, const double *moved5, double *target5, int64_t ntri, const int *tris,
                   double omega, int64_t *fallback) {
    return orc_remesh_keyed(n, moved5, target5, ntri, tris, NULL, omega, fallback);
}

/* ------------------------------------------------------------------ AMR */

/* amr.h:13-178 amr on flat arrays.  Triangles are visited in index order
 * while the count grows (children appended during the pass are visited in
 * the same pass; the first child keeps the parent's index and is not).  A
 * triangle is split in four when its vorticity range exceeds vtol or its
 * circulation A |z1 + z2 + z3| / 3 exceeds ctol (the reference hard-codes
 * 0.2 and 0.0025).  Edge midpoints (unprojected averages of all five state
 * components) are shared through the parent pairs (check_in_vec3: the first
 * point whose pair is (min, max)); areas move A/6 from each corner to each
 * midpoint.  The reference's vert_tris lists are kept as one key per
 * triangle corner: a list is its triangles in increasing key order (initial
 * lists by triangle index; appended entries 2^40 + 9 s + slot, s the
 * refinement's running number).  parent has two ints per point, (0, 0) for
 * primitive points.  Returns 0, or -1 when max_points or max_tris would be
 * exceeded (undefined behaviour in the reference; arrays then partly
 * updated).  Nothing happens when *n >= max_points (as the reference). */
#define AMR_KEY_APPEND ((uint64_t)1 << 40)
static int amr_find_parent(const int *parent, int64_t n, int a, int b) {
    for (int64_t i = 0; i < n; i++)
        if (parent[2 * i] == a && parent[2 * i + 1] == b) return (int)i;
    return -1;
}

int orc_amr(int64_t *n_io, int64_t max_points, double *state5, double *area, int64_t *ntri_io, int64_t max_tris,
            int *tris, uint64_t *keys, int *parent, uint64_t *seq_io, double vtol, double ctol) {
    int64_t n = *n_io, ntri = *ntri_io;
    uint64_t seq = *seq_io;
    int rc = 0;
    if (n >= max_points) return 0;
    for (int64_t i = 0; i < ntri; i++) {
        const int iv1 = tris[3 * i], iv2 = tris[3 * i + 1], iv3 = tris[3 * i + 2];
        const double vor1 = state5[5 * (int64_t)iv1 + 3], vor2 = state5[5 * (int64_t)iv2 + 3],
                     vor3 = state5[5 * (int64_t)iv3 + 3];
        double mx = (vor2 < vor3) ? vor3 : vor2; /* std::max(vor1, std::max(vor2, vor3)) */
        mx = (vor1 < mx) ? mx : vor1;
        double mn = (vor3 < vor2) ? vor3 : vor2; /* std::min */
        mn = (mn < vor1) ? mn : vor1;
        const double A = orc_sphere_tri_area(state5 + 5 * (int64_t)iv1, state5 + 5 * (int64_t)iv2,
                                             state5 + 5 * (int64_t)iv3, 1.0);
        const double circ = A * fabs(vor1 + vor2 + vor3) / 3.0;
        if (!((mx - mn) > vtol || circ > ctol)) continue;
        area[iv1] -= A / 6.0;
        area[iv2] -= A / 6.0;
        area[iv3] -= A / 6.0;
        const int ea[3] = {iv1, iv2, iv3}, eb[3] = {iv2, iv3, iv1}; /* v12 = v1 + v2, v23 = v2 + v3, v31 = v3 + v1 */
        int m[3];
        for (int k = 0; k < 3; k++) {
            const int lo = ea[k] < eb[k] ? ea[k] : eb[k], hi = ea[k] < eb[k] ? eb[k] : ea[k];
            m[k] = amr_find_parent(parent, n, lo, hi);
        }
        for (int k = 0; k < 3; k++) {
            const int lo = ea[k] < eb[k] ? ea[k] : eb[k], hi = ea[k] < eb[k] ? eb[k] : ea[k];
            if (m[k] == -1) {
                if (n >= max_points) { rc = -1; goto done; }
                m[k] = (int)n;
                for (int c = 0; c < 5; c++) {
                    double v = state5[5 * (int64_t)ea[k] + c];
                    v += state5[5 * (int64_t)eb[k] + c];
                    state5[5 * n + c] = v * 0.5;
                }
                area[n] = A / 6.0;
                parent[2 * n] = lo;
                parent[2 * n + 1] = hi;
                n++;
            } else {
                area[m[k]] += A / 6.0;
            }
        }
        if (ntri + 3 > max_tris) { rc = -1; goto done; }
        {
            const int m12 = m[0], m23 = m[1], m31 = m[2];
            const uint64_t k1 = keys[3 * i], k2 = keys[3 * i + 1], k3 = keys[3 * i + 2];
            const uint64_t b = AMR_KEY_APPEND + 9 * seq;
            const int64_t t2 = ntri, t3 = ntri + 1, t4 = ntri + 2;
            tris[3 * i] = iv1; tris[3 * i + 1] = m12; tris[3 * i + 2] = m31;
            keys[3 * i] = k1; keys[3 * i + 1] = b + 0; keys[3 * i + 2] = b + 6;
            tris[3 * t2] = iv2; tris[3 * t2 + 1] = m12; tris[3 * t2 + 2] = m23;
            keys[3 * t2] = k2; keys[3 * t2 + 1] = b + 1; keys[3 * t2 + 2] = b + 3;
            tris[3 * t3] = iv3; tris[3 * t3 + 1] = m31; tris[3 * t3 + 2] = m23;
            keys[3 * t3] = k3; keys[3 * t3 + 1] = b + 7; keys[3 * t3 + 2] = b + 4;
            tris[3 * t4] = m12; tris[3 * t4 + 1] = m23; tris[3 * t4 + 2] = m31;
            keys[3 * t4] = b + 2; keys[3 * t4 + 1] = b + 5; keys[3 * t4 + 2] = b + 8;
            ntri += 3;
            seq++;
        }
    }
done:
    *n_io = n;
    *ntri_io = ntri;
    *seq_io = seq;
    return rc;
}
