// Drop-in check: the reference's RK4 loop shape (new_dynamics.cpp:281-340)
// driven through include/fss_rhs_func.hpp's rhs_func with a struct that has
// the fields of the reference's run_information (struct_list.h:50-102).
// Prints "dropin ok <rel-l2 fast vs direct>" and exits 0 on success.
#include <cmath>
#include <cstdio>
#include <vector>

#include "fss_rhs_func.hpp"

struct run_information {  // the fields rhs_func reads, same names and types
    bool use_fast = false;
    int point_count = 0;
    int tree_levels = 1;
    double theta = 0.7;
    int many_count = 10;
    int degree = 2;
};

int main() {
    const int level = 5;
    int64_t nv, nf;
    if (fss_icos_counts(level, &nv, &nf) != FSS_OK) return 2;
    std::vector<double> xyz(3 * nv), state(5 * nv, 0.0), area(nv);
    std::vector<int32_t> faces(3 * nf);
    fss_icos_grid(level, xyz.data(), faces.data());
    for (int64_t i = 0; i < nv; i++)
        for (int k = 0; k < 3; k++) state[5 * i + k] = xyz[3 * i + k];
    fss_area_init(nv, state.data(), nf, faces.data(), area.data());
    fss_vorticity_rh4_ref(nv, state.data());

    run_information cfg;
    cfg.point_count = (int)nv;
    std::vector<double> direct(5 * nv), fast(5 * nv);
    rhs_func(direct, state, area, 2 * M_PI, cfg);
    cfg.use_fast = true;
    cfg.tree_levels = 3;
    cfg.many_count = 45;
    cfg.degree = 8;
    rhs_func(fast, state, area, 2 * M_PI, cfg);
    rhs_func(fast, state, area, 2 * M_PI, cfg);  // second call reuses the tree
    double num = 0, den = 0;
    for (int64_t i = 0; i < nv; i++)
        for (int k = 0; k < 3; k++) {
            const double d = fast[5 * i + k] - direct[5 * i + k];
            num += d * d;
            den += direct[5 * i + k] * direct[5 * i + k];
        }
    const double rel = std::sqrt(num / den);
    std::printf("dropin ok %.3e\n", rel);
    return rel < 1e-5 ? 0 : 1;
}
