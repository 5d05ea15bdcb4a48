// Drop-in check: the reference's own run_information (struct_list.h:50-102)
// and vector helpers (helpers.h: scalar_mult, vec_add, project_points),
// with include/fss_rhs_func.hpp's rhs_func in place of rhs_eval.h's, in the
// RK4 loop of new_dynamics.cpp:170-229 (four rhs_func calls per step, stage
// states projected onto the sphere).  Built by oracle/Makefile (target
// dropin) against the reference's headers where they lie.
//
//   dropin <level> <out.f64>
//
// On the level's icosahedral grid with the reference's RH4 field, writes as
// float64, one after another: modify of the first rhs_func call with
// use_fast = false (FP64, as the reference); the state after two RK4 steps
// of dt = 0.01 with that evaluator; modify with use_fast = true (treecode,
// degree 8, 3 tree levels, FP64); modify with use_fast = true in mixed
// precision.  Each is 5 doubles per particle.  Prints "dropin ok" and exits 0
// when every call succeeded.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "helpers.h"
#include "struct_list.h"

#include "fss_rhs_func.hpp"

static void rk4_step(vector<double>& curr_state, vector<double>& area, double omega, double delta_t,
                     run_information& config1) {
    const int n = config1.point_count;
    vector<double> c_1(5 * n), c_2(5 * n), c_3(5 * n), c_4(5 * n), c1234;
    vector<double> intermediate_1, intermediate_2, intermediate_3;
    rhs_func(c_1, curr_state, area, omega, config1);
    intermediate_1 = c_1;
    scalar_mult(intermediate_1, delta_t / 2);
    vec_add(intermediate_1, curr_state);
    project_points(intermediate_1, n, omega);
    rhs_func(c_2, intermediate_1, area, omega, config1);
    intermediate_2 = c_2;
    scalar_mult(intermediate_2, delta_t / 2);
    vec_add(intermediate_2, curr_state);
    project_points(intermediate_2, n, omega);
    rhs_func(c_3, intermediate_2, area, omega, config1);
    intermediate_3 = c_3;
    scalar_mult(intermediate_3, delta_t);
    vec_add(intermediate_3, curr_state);
    project_points(intermediate_3, n, omega);
    rhs_func(c_4, intermediate_3, area, omega, config1);
    c1234 = c_1;
    scalar_mult(c_2, 2);
    vec_add(c1234, c_2);
    scalar_mult(c_3, 2);
    vec_add(c1234, c_3);
    vec_add(c1234, c_4);
    scalar_mult(c1234, delta_t / 6);
    vec_add(curr_state, c1234);
    project_points(curr_state, n, omega);
}

int main(int argc, char** argv) {
    if (argc < 3) {
        std::fprintf(stderr, "usage: dropin <level> <out.f64>\n");
        return 2;
    }
    const int level = std::atoi(argv[1]);
    int64_t nv, nf;
    if (fss_icos_counts(level, &nv, &nf) != FSS_OK) return 2;
    std::vector<double> xyz(3 * nv);
    std::vector<int32_t> faces(3 * nf);
    fss_icos_grid(level, xyz.data(), faces.data());

    run_information config1;
    config1.point_count = (int)nv;
    vector<double> state(5 * nv, 0.0), area(nv);
    for (int64_t i = 0; i < nv; i++)
        for (int k = 0; k < 3; k++) state[5 * i + k] = xyz[3 * i + k];
    fss_area_init(nv, state.data(), nf, faces.data(), area.data());
    fss_vorticity_rh4_ref(nv, state.data());
    const double omega = 2 * M_PI;

    FILE* f = std::fopen(argv[2], "wb");
    if (!f) return 2;
    try {
        vector<double> modify(5 * nv);
        config1.use_fast = false;
        rhs_func(modify, state, area, omega, config1);
        std::fwrite(modify.data(), sizeof(double), modify.size(), f);

        vector<double> s = state;
        rk4_step(s, area, omega, 0.01, config1);
        rk4_step(s, area, omega, 0.01, config1);
        std::fwrite(s.data(), sizeof(double), s.size(), f);

        config1.use_fast = true;
        config1.tree_levels = 3;
        config1.many_count = 45;
        config1.degree = 8;
        config1.theta = 0.7;
        rhs_func(modify, state, area, omega, config1);
        rhs_func(modify, state, area, omega, config1);  // second call reuses the tree
        std::fwrite(modify.data(), sizeof(double), modify.size(), f);

        fss_dropin::set_precision(FSS_PREC_MIXED);
        rhs_func(modify, state, area, omega, config1);
        std::fwrite(modify.data(), sizeof(double), modify.size(), f);
    } catch (const std::exception& e) {
        std::fclose(f);
        std::fprintf(stderr, "dropin failed: %s\n", e.what());
        return 1;
    }
    std::fclose(f);
    std::printf("dropin ok\n");
    return 0;
}
