// geometry.h -- host icosahedral tree geometry and synthetic inputs.
#pragma once
#include <cstdint>
#include <vector>

#include "fss_internal.h"

namespace fss {

// Tree geometry of levels 0..tree_levels-1 (icos_utils.h:15 icos_init):
// verts (3 doubles each), tri_verts (3 ids per face), tri_info (circumcentre
// xyz + circumradius per face), faces of level l at [lev_off[l], lev_off[l+1]).
struct TreeGeometry {
    int tree_levels = 0;
    std::vector<double> verts;
    std::vector<int32_t> tri_verts;
    std::vector<double> tri_info;
    std::vector<int64_t> lev_off;
    std::vector<NodeGeom> node;  // per face: barycentric frame
    int64_t level_count(int l) const { return lev_off[l + 1] - lev_off[l]; }
};

TreeGeometry build_tree_geometry(int tree_levels);
void icos_grid(int level, std::vector<double>& xyz, std::vector<int32_t>& faces);
void area_init(int64_t n, const double* s5, int64_t nf, const int32_t* faces, double* area);
void vorticity_rh4_ref(int64_t n, double* s5);
void vorticity_rh_vortices(int64_t n, double* s5, const double* area, double amp, int nvort, double width,
                           uint64_t seed);
double great_circ_dist(const double* p1, const double* p2, double radius);
void tri_center(const double* p1, const double* p2, const double* p3, double radius, double* c);
double tri_radius(const double* p1, const double* p2, const double* p3, const double* c);

}  // namespace fss
