// amr_internal.h -- the AMR handle behind fss_amr (private to the library).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "kernels.h"

struct fss_amr {
    int dev = 0;
    cudaStream_t st = nullptr;
    int64_t n = 0, ntri = 0, max_points = 0, max_tris = 0;
    uint64_t seq = 0;  // refinements so far (append keys)
    bool broken = false;
    // mesh
    fss::DBuf state5, area, tris, keys, parent, hkeys, hvals, err;
    int64_t hmask = 0;
    // one pass
    fss::DBuf flag, rank, tarea, refined, occ_slot, cflag, crank, part;
    fss::DBuf rec_v, rec_d, rec_k, sort_tmp, sort_perm, sort_perm_tmp, sort_hist;
    // remesh on the current mesh
    fss::DBuf moved, target, off, adj;
    bool adj_ok = false;
    fss::RemeshScratch rs;
    ~fss_amr() {
        if (st) cudaStreamDestroy(st);
    }
};

namespace fss {
// One amr() pass on the handle's device state (host arrays untouched).
// On an error status the device arrays are partly updated and the caller
// must treat the handle as unusable.
int amr_refine_device(fss_amr* a, double vtol, double ctol);
}  // namespace fss
