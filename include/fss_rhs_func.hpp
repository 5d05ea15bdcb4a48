// fss_rhs_func.hpp -- header-only C++ drop-in for the reference's right-hand
// side (cygnari/fast-sphere-sum Old-BVE-code/rhs_eval.h:47-56):
//
//   void rhs_func(vector<double>& modify, vector<double>& curr_state,
//                 vector<double>& area, double omega, run_information& config1);
//
// Include this header in place of rhs_eval.h and link libfss.so.  It reads the
// fields the reference's evaluators read from run_information -- use_fast,
// point_count, tree_levels, theta, many_count, degree -- and evaluates on the
// GPU through the C ABI of fss.h.  As in the reference (new_dynamics.cpp:87-88),
// the tree is built from the particles of the first call and kept for later
// calls with the same settings; a change of any setting or of point_count
// rebuilds it.  Errors throw std::runtime_error (the reference has no error
// path; it prints LAPACK info and continues).
//
// Precision: FP64 throughout by default, as the reference's rhs_func.  A
// caller that wants the mixed-precision evaluator (FP32 interactions with
// Kahan-compensated sums, about 1e-7 relative error) selects it with
// fss_dropin::set_precision(FSS_PREC_MIXED) before the call, or compiles with
// -DFSS_DROPIN_PRECISION=FSS_PREC_MIXED.
#pragma once

#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "fss.h"

#ifndef FSS_DROPIN_PRECISION
#define FSS_DROPIN_PRECISION FSS_PREC_FP64
#endif

namespace fss_dropin {

struct Settings {
    bool use_fast = false;
    int point_count = 0, tree_levels = 0, many_count = -1, degree = 8;
    double theta = 0.7;
    int precision = FSS_DROPIN_PRECISION;
    bool operator==(const Settings& o) const {
        return use_fast == o.use_fast && point_count == o.point_count && tree_levels == o.tree_levels &&
               many_count == o.many_count && degree == o.degree && theta == o.theta && precision == o.precision;
    }
};

// Precision of later rhs_func calls on this thread (fss_precision).
inline int& precision_setting() {
    thread_local int p = FSS_DROPIN_PRECISION;
    return p;
}
inline void set_precision(int p) {
    if (p != FSS_PREC_FP64 && p != FSS_PREC_MIXED) throw std::invalid_argument("fss: unknown precision");
    precision_setting() = p;
}

struct Ctx {
    fss_ctx* h = nullptr;
    Settings s;
    ~Ctx() { if (h) fss_destroy(h); }
};

inline void check(int rc, fss_ctx* h) {
    if (rc != FSS_OK) throw std::runtime_error(std::string("fss: ") + fss_last_error(h));
}

// One context per thread, rebuilt when the settings change.
inline Ctx& context(const Settings& s, const double* state5, const double* area) {
    thread_local std::unique_ptr<Ctx> ctx;
    if (!ctx || !(ctx->s == s)) {
        ctx.reset(new Ctx());
        fss_config cfg;
        fss_config_init(&cfg);
        cfg.precision = s.precision;
        cfg.method = s.use_fast ? FSS_METHOD_TREECODE : FSS_METHOD_DIRECT;
        cfg.tree_levels = s.tree_levels;
        cfg.theta = s.theta;
        cfg.many_count = s.many_count;
        cfg.degree = s.degree;
        check(fss_create(&cfg, &ctx->h), nullptr);
        ctx->s = s;
        check(fss_set_particles(ctx->h, s.point_count, state5, area), ctx->h);
    }
    return *ctx;
}

}  // namespace fss_dropin

// rhs_eval.h:47 rhs_func.  RunInfo is the reference's run_information (or any
// type with the same fields).
template <class RunInfo>
void rhs_func(std::vector<double>& modify, std::vector<double>& curr_state, std::vector<double>& area, double omega,
              RunInfo& config1) {
    fss_dropin::Settings s;
    s.use_fast = config1.use_fast;
    s.point_count = config1.point_count;
    s.tree_levels = config1.use_fast ? config1.tree_levels : 0;
    s.theta = config1.theta;
    s.many_count = config1.use_fast ? config1.many_count : -1;
    s.degree = (config1.use_fast && config1.degree > 0) ? config1.degree : 8;
    s.precision = fss_dropin::precision_setting();
    if ((int64_t)curr_state.size() < 5 * (int64_t)s.point_count || (int64_t)area.size() < s.point_count)
        throw std::runtime_error("fss: state/area shorter than point_count");
    modify.resize(curr_state.size());
    fss_dropin::Ctx& c = fss_dropin::context(s, curr_state.data(), area.data());
    fss_dropin::check(fss_rhs(c.h, curr_state.data(), area.data(), omega, modify.data(), nullptr), c.h);
}
