// geometry.cpp -- host-side icosahedral geometry and synthetic inputs.
//
// Compiled with -ffp-contract=off: the tree geometry feeds the bit-exact
// particle assignment and MAC, so every expression keeps the operation order
// of the reference (cygnari/fast-sphere-sum Old-BVE-code/helpers.h and
// icos_utils.h), and no multiply-add may be fused.
#include "geometry.h"

#include <cmath>
#include <cstring>
#include <random>
#include <unordered_map>

namespace fss {

static inline double dot3(const double* x, const double* y) {
    double s = 0;  // helpers.h:23-28: sequential from 0
    s += x[0] * y[0];
    s += x[1] * y[1];
    s += x[2] * y[2];
    return s;
}
static inline double norm3(const double* x) { return std::sqrt(dot3(x, x)); }

// helpers.h:82-85 project_to_sphere (p *= radius / |p|)
static inline void project(double* p, double radius) {
    double n = norm3(p);
    for (int i = 0; i < 3; i++) p[i] *= radius / n;
}

// helpers.h:183-196 tri_center (circumcentre, projected) with tri_sides
void tri_center(const double* p1, const double* p2, const double* p3, double radius, double* c) {
    double p23[3], p31[3], p12[3];
    for (int i = 0; i < 3; i++) {
        p23[i] = p2[i] - p3[i];
        p31[i] = p3[i] - p1[i];
        p12[i] = p1[i] - p2[i];
    }
    const double a = norm3(p23), b = norm3(p31), cc = norm3(p12);
    auto poly = [](double x, double y, double z) { return x * x + y * y - z * z; };
    const double scaling = (a + b + cc) * (a + b - cc) * (a - b + cc) * (b + cc - a);
    const double k1 = a * a * poly(b, cc, a) / scaling;
    const double k2 = b * b * poly(cc, a, b) / scaling;
    const double k3 = cc * cc * poly(a, b, cc) / scaling;
    for (int k = 0; k < 3; k++) c[k] = k1 * p1[k] + k2 * p2[k] + k3 * p3[k];
    project(c, radius);
}

// helpers.h:198-209 tri_radius (largest vertex distance from the centre)
double tri_radius(const double* p1, const double* p2, const double* p3, const double* c) {
    double d[3][3];
    for (int i = 0; i < 3; i++) {
        d[0][i] = p1[i] - c[i];
        d[1][i] = p2[i] - c[i];
        d[2][i] = p3[i] - c[i];
    }
    const double r1 = norm3(d[0]), r2 = norm3(d[1]), r3 = norm3(d[2]);
    const double m = (r1 < r2) ? r2 : r1;
    return (m < r3) ? r3 : m;
}

// helpers.h:211-215 great_circ_dist
double great_circ_dist(const double* p1, const double* p2, double radius) {
    const double s = dot3(p1, p2) / (norm3(p1) * norm3(p2));
    const double lo = (s < -1.0) ? -1.0 : s;
    const double cl = (1.0 < lo) ? 1.0 : lo;
    return std::acos(cl) * radius;
}

// icos_utils.h:15-133 icos_init.  Midpoints are de-duplicated by their edge
// (the pair of parent vertex ids) instead of the reference's linear scan for
// equal coordinates: a midpoint is computed identically from either side of
// its edge and distinct edges give distinct points, so the first-insertion
// order -- v12, v31, v23 per parent face, faces in order -- is the same.
static void icos_build(int levels, double radius, bool with_info, std::vector<double>& verts,
                       std::vector<int32_t>& tri_verts, std::vector<double>& tri_info,
                       std::vector<int64_t>& lev_off) {
    int64_t nf_total = 0, nf = 20;
    lev_off.assign(levels + 2, 0);
    for (int l = 0; l <= levels; l++) {
        lev_off[l] = nf_total;
        nf_total += nf;
        nf *= 4;
    }
    lev_off[levels + 1] = nf_total;
    const int64_t nv_final = 10 * (int64_t(1) << (2 * levels)) + 2;
    verts.assign(3 * nv_final, 0.0);
    tri_verts.assign(3 * nf_total, 0);
    if (with_info) tri_info.assign(4 * nf_total, 0.0);

    const double phi = (1 + std::sqrt(5)) / 2;
    const double base[12][3] = {{0, 1, phi}, {0, -1, phi}, {0, 1, -phi}, {0, -1, -phi},
                                {1, phi, 0}, {1, -phi, 0}, {-1, phi, 0}, {-1, -phi, 0},
                                {phi, 0, 1}, {phi, 0, -1}, {-phi, 0, 1}, {-phi, 0, -1}};
    int64_t nv = 0;
    for (int i = 0; i < 12; i++, nv++) {  // helpers.h:87-92 project_to_sphere_2
        const double n = norm3(base[i]);
        for (int k = 0; k < 3; k++) verts[3 * nv + k] = radius * base[i][k] / n;
    }
    static const int faces1[20][3] = {{1, 2, 9},  {1, 2, 11}, {1, 5, 7},  {1, 5, 9},   {1, 7, 11},
                                      {2, 6, 8},  {2, 6, 9},  {2, 8, 11}, {3, 4, 10},  {3, 4, 12},
                                      {3, 5, 7},  {3, 5, 10}, {3, 7, 12}, {4, 6, 8},   {4, 6, 10},
                                      {4, 8, 12}, {5, 9, 10}, {6, 9, 10}, {7, 11, 12}, {8, 11, 12}};
    for (int i = 0; i < 20; i++) {
        for (int j = 0; j < 3; j++) tri_verts[3 * i + j] = faces1[i][j] - 1;
        if (with_info) {
            const double* v1 = &verts[3 * tri_verts[3 * i]];
            const double* v2 = &verts[3 * tri_verts[3 * i + 1]];
            const double* v3 = &verts[3 * tri_verts[3 * i + 2]];
            double* ti = &tri_info[4 * i];
            tri_center(v1, v2, v3, radius, ti);
            ti[3] = tri_radius(v1, v2, v3, ti);
        }
    }
    std::unordered_map<uint64_t, int32_t> edge;
    edge.reserve(size_t(nv_final * 1.3));
    auto mid = [&](int32_t a, int32_t b, const double* va, const double* vb) -> int32_t {
        const uint64_t key = (a < b) ? (uint64_t(a) << 32 | uint32_t(b)) : (uint64_t(b) << 32 | uint32_t(a));
        auto it = edge.find(key);
        if (it != edge.end()) return it->second;
        double m[3];
        for (int k = 0; k < 3; k++) m[k] = va[k] + vb[k];
        for (int k = 0; k < 3; k++) m[k] *= 0.5;
        project(m, radius);
        const int32_t id = int32_t(nv++);
        std::memcpy(&verts[3 * int64_t(id)], m, 24);
        edge.emplace(key, id);
        return id;
    };
    for (int l = 0; l < levels; l++) {
        edge.clear();
        const int64_t off = lev_off[l], noff = lev_off[l + 1], cnt = noff - off;
        for (int64_t j = 0; j < cnt; j++) {
            const int32_t iv1 = tri_verts[3 * (off + j)], iv2 = tri_verts[3 * (off + j) + 1],
                          iv3 = tri_verts[3 * (off + j) + 2];
            double v1[3], v2[3], v3[3];
            std::memcpy(v1, &verts[3 * int64_t(iv1)], 24);
            std::memcpy(v2, &verts[3 * int64_t(iv2)], 24);
            std::memcpy(v3, &verts[3 * int64_t(iv3)], 24);
            // the reference checks v12, v31, v23 and appends in that order
            const int32_t iv12 = mid(iv1, iv2, v1, v2);
            const int32_t iv13 = mid(iv3, iv1, v3, v1);
            const int32_t iv23 = mid(iv2, iv3, v2, v3);
            int32_t* c = &tri_verts[3 * (noff + 4 * j)];
            c[0] = iv1;  c[1] = iv13; c[2] = iv12;
            c[3] = iv3;  c[4] = iv23; c[5] = iv13;
            c[6] = iv2;  c[7] = iv12; c[8] = iv23;
            c[9] = iv12; c[10] = iv13; c[11] = iv23;
            if (with_info) {
                const double* v12 = &verts[3 * int64_t(iv12)];
                const double* v31 = &verts[3 * int64_t(iv13)];
                const double* v23 = &verts[3 * int64_t(iv23)];
                double* ti = &tri_info[4 * (noff + 4 * j)];
                tri_center(v1, v12, v31, radius, ti);
                ti[3] = tri_radius(v1, v12, v31, ti);
                tri_center(v3, v23, v31, radius, ti + 4);
                ti[7] = tri_radius(v3, v23, v31, ti + 4);
                tri_center(v2, v12, v23, radius, ti + 8);
                ti[11] = tri_radius(v2, v12, v23, ti + 8);
                tri_center(v12, v31, v23, radius, ti + 12);
                ti[15] = tri_radius(v12, v31, v23, ti + 12);
            }
        }
    }
}

TreeGeometry build_tree_geometry(int tree_levels) {
    TreeGeometry g;
    g.tree_levels = tree_levels;
    icos_build(tree_levels - 1, 1.0, true, g.verts, g.tri_verts, g.tri_info, g.lev_off);
    // the reference also refines once more (icos_init(tree_levels)); those
    // faces are never used by points_assign or tree_traverse.
    const int64_t nfaces = g.lev_off[tree_levels];
    g.node.resize(nfaces);
    for (int64_t f = 0; f < nfaces; f++) {
        const double* v[3] = {&g.verts[3 * int64_t(g.tri_verts[3 * f])], &g.verts[3 * int64_t(g.tri_verts[3 * f + 1])],
                              &g.verts[3 * int64_t(g.tri_verts[3 * f + 2])]};
        // M = [v1 v2 v3] (columns); invert by cofactors in FP64.
        const double a = v[0][0], b = v[1][0], c = v[2][0];
        const double d = v[0][1], e = v[1][1], f2 = v[2][1];
        const double gg = v[0][2], h = v[1][2], i = v[2][2];
        const double A = e * i - f2 * h, B = -(d * i - f2 * gg), C = d * h - e * gg;
        const double det = a * A + b * B + c * C;
        NodeGeom& ng = g.node[f];
        ng.minv[0] = A / det;                 ng.minv[1] = -(b * i - c * h) / det; ng.minv[2] = (b * f2 - c * e) / det;
        ng.minv[3] = B / det;                 ng.minv[4] = (a * i - c * gg) / det;  ng.minv[5] = -(a * f2 - c * d) / det;
        ng.minv[6] = C / det;                 ng.minv[7] = -(a * h - b * gg) / det; ng.minv[8] = (a * e - b * d) / det;
        ng.cx = g.tri_info[4 * f];
        ng.cy = g.tri_info[4 * f + 1];
        ng.cz = g.tri_info[4 * f + 2];
    }
    return g;
}

void icos_grid(int level, std::vector<double>& xyz, std::vector<int32_t>& faces) {
    std::vector<double> info;
    std::vector<int32_t> tv;
    std::vector<int64_t> off;
    icos_build(level, 1.0, false, xyz, tv, info, off);
    faces.assign(tv.begin() + 3 * off[level], tv.begin() + 3 * off[level + 1]);
}

// helpers.h:94-115 sphere_tri_area
static double sphere_tri_area(const double* p1, const double* p2, const double* p3) {
    double p1n[3], p2n[3], p3n[3];
    for (int i = 0; i < 3; i++) {
        p2n[i] = p2[i] - p3[i];
        p3n[i] = p3[i] - p1[i];
        p1n[i] = p1[i] - p2[i];
    }
    const double a = std::acos(1 - 0.5 * dot3(p2n, p2n));
    const double b = std::acos(1 - 0.5 * dot3(p3n, p3n));
    const double c = std::acos(1 - 0.5 * dot3(p1n, p1n));
    const double s = (a + b + c) / 2;
    const double z = std::tan(s / 2) * std::tan((s - a) / 2) * std::tan((s - b) / 2) * std::tan((s - c) / 2);
    return 4 * 1.0 * 1.0 * std::atan(std::sqrt(z));
}

// helpers.h:344-360 area_init
void area_init(int64_t n, const double* s5, int64_t nf, const int32_t* faces, double* area) {
    for (int64_t i = 0; i < n; i++) area[i] = 0;
    for (int64_t t = 0; t < nf; t++) {
        const int64_t i1 = faces[3 * t], i2 = faces[3 * t + 1], i3 = faces[3 * t + 2];
        const double a = sphere_tri_area(s5 + 5 * i1, s5 + 5 * i2, s5 + 5 * i3);
        area[i1] += a / 3.0;
        area[i2] += a / 3.0;
        area[i3] += a / 3.0;
    }
}

// helpers.h:117-124 lat_lon
static inline void lat_lon(const double* p, double* lat, double* lon) {
    const double x = p[0], y = p[1], z = p[2];
    *lat = M_PI / 2 - std::atan2(std::sqrt(x * x + y * y), z);
    *lon = std::atan2(y, x);
}

// vorticity_functions.h:13-24 rossby_haurwitz_4
void vorticity_rh4_ref(int64_t n, double* s5) {
    for (int64_t i = 0; i < n; i++) {
        double lat, lon;
        lat_lon(s5 + 5 * i, &lat, &lon);
        s5[5 * i + 4] = 2 + lat;
        s5[5 * i + 3] = 2 * M_PI * std::sin(lat) / 7.0 +
                        30.0 * std::sin(lat) * std::pow(std::cos(lat), 4) * std::cos(4 * lon);
    }
}

// Rossby-Haurwitz wave R=4 plus seeded Gaussian vortices (synthetic input).
void vorticity_rh_vortices(int64_t n, double* s5, const double* area, double amp, int nvort, double width,
                           uint64_t seed) {
    std::mt19937_64 rng(seed);
    auto uni = [&]() { return double(rng() >> 11) * (1.0 / 9007199254740992.0); };  // [0, 1)
    std::vector<double> cx(nvort), cy(nvort), cz(nvort), ca(nvort);
    for (int v = 0; v < nvort; v++) {
        const double z = 2 * uni() - 1, lon = 2 * M_PI * uni();
        const double r = std::sqrt(std::max(0.0, 1 - z * z));
        cx[v] = r * std::cos(lon);
        cy[v] = r * std::sin(lon);
        cz[v] = z;
        // Box-Muller: amplitude ~ N(0, variance 2 pi^2)
        const double u1 = 1.0 - uni(), u2 = uni();
        ca[v] = std::sqrt(2 * M_PI * M_PI) * std::sqrt(-2 * std::log(u1)) * std::cos(2 * M_PI * u2);
    }
    const int R = 4;
    const double w = amp, K = amp;
    double tot = 0, atot = 0;
    for (int64_t i = 0; i < n; i++) {
        double lat, lon;
        const double* p = s5 + 5 * i;
        lat_lon(p, &lat, &lon);
        double z = 2 * w * std::sin(lat) -
                   K * (R + 1) * (R + 2) * std::pow(std::cos(lat), R) * std::sin(lat) * std::cos(R * lon);
        for (int v = 0; v < nvort; v++) {
            double d = p[0] * cx[v] + p[1] * cy[v] + p[2] * cz[v];
            d = std::acos(std::min(1.0, std::max(-1.0, d)));
            z += ca[v] * std::exp(-(d / width) * (d / width));
        }
        s5[5 * i + 3] = z;
        s5[5 * i + 4] = 2 + lat;
        if (area) {
            tot += z * area[i];
            atot += area[i];
        }
    }
    if (area && atot > 0) {
        const double mean = tot / atot;
        for (int64_t i = 0; i < n; i++) s5[5 * i + 3] -= mean;
    }
}

}  // namespace fss
