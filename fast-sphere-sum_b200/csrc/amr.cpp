// amr.cpp -- the AMR handle: the mesh (triangles, per-corner adjacency
// keys, parent pairs) on the device, refined by the generation kernels of
// k_amr.cu (amr.h:13-178 amr), and the remesh step on that mesh
// (remesh.h:109 regrid_points2 with the vert_tris lists amr() keeps).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "amr_internal.h"
#include "fss.h"
#include "kernels.h"

namespace fss {
void set_last_error(const std::string& msg);
}

using namespace fss;

namespace {

int afail(int code, const std::string& m) {
    set_last_error(m);
    return code;
}

#define ACU(call)                                                                                        \
    do {                                                                                                 \
        cudaError_t e_ = (call);                                                                         \
        if (e_ != cudaSuccess)                                                                           \
            return afail(e_ == cudaErrorMemoryAllocation ? FSS_ERR_NOMEM : FSS_ERR_CUDA,                 \
                         std::string(#call) + ": " + cudaGetErrorString(e_));                            \
    } while (0)

int64_t pow2_at_least(int64_t x) {
    int64_t p = 1;
    while (p < x) p <<= 1;
    return p;
}

int bits_for(int64_t n) {
    int b = 8;
    while (b < 32 && (int64_t(1) << b) < n) b += 8;
    return b;
}

// Total of an exclusive scan: rank + flag of the last entry (synchronises).
int scan_total(fss_amr* a, const uint32_t* rank, const uint32_t* flag, int64_t m, int64_t* total) {
    uint32_t h[2] = {0, 0};
    ACU(cudaMemcpyAsync(h, rank + (m - 1), sizeof(uint32_t), cudaMemcpyDeviceToHost, a->st));
    ACU(cudaMemcpyAsync(h + 1, flag + (m - 1), sizeof(uint32_t), cudaMemcpyDeviceToHost, a->st));
    ACU(cudaStreamSynchronize(a->st));
    *total = int64_t(h[0]) + h[1];
    return FSS_OK;
}

}  // namespace

// The whole pass on the device state; host buffers are not touched.
int fss::amr_refine_device(fss_amr* a, double vtol, double ctol) {
    cudaStream_t st = a->st;
    int64_t n = a->n, q0 = 0, q1 = a->ntri, nrec = 0;
    uint64_t seq = a->seq;
    // every refinement appends three triangles: records are bounded by the
    // triangle capacity
    const int64_t max_ref = std::max<int64_t>((a->max_tris - a->ntri) / 3, 1);
    ACU(a->rec_v.ensure(sizeof(uint32_t) * 6 * size_t(max_ref)));
    ACU(a->rec_d.ensure(sizeof(double) * 6 * size_t(max_ref)));
    ACU(a->rec_k.ensure(sizeof(uint8_t) * 6 * size_t(max_ref)));
    int* derr = a->err.as<int>();
    ACU(cudaMemsetAsync(derr, 0, sizeof(int), st));
    while (q1 > q0) {
        const int64_t m = q1 - q0;
        ACU(a->flag.ensure(sizeof(uint32_t) * size_t(m)));
        ACU(a->rank.ensure(sizeof(uint32_t) * size_t(m)));
        ACU(a->tarea.ensure(sizeof(double) * size_t(m)));
        ACU(a->part.ensure(sizeof(uint32_t) * size_t(scan_part_words(3 * m))));
        amr_test(st, q0, m, a->tris.as<int32_t>(), a->state5.as<double>(), vtol, ctol, a->flag.as<uint32_t>(),
                 a->rank.as<uint32_t>(), a->tarea.as<double>());
        launch_scan_u32(st, a->rank.as<uint32_t>(), m, a->part.as<uint32_t>());
        int64_t R = 0;
        if (int rc = scan_total(a, a->rank.as<uint32_t>(), a->flag.as<uint32_t>(), m, &R)) return rc;
        if (R == 0) break;
        if (q1 + 3 * R > a->max_tris || nrec + 6 * R > 6 * max_ref)
            return afail(FSS_ERR_CAPACITY, "amr: more triangles than the handle's max_tris");
        ACU(a->refined.ensure(sizeof(int32_t) * size_t(R)));
        ACU(a->occ_slot.ensure(sizeof(int64_t) * 3 * size_t(R)));
        ACU(a->cflag.ensure(sizeof(uint32_t) * 3 * size_t(R)));
        ACU(a->crank.ensure(sizeof(uint32_t) * 3 * size_t(R)));
        amr_edges(st, q0, m, a->flag.as<uint32_t>(), a->rank.as<uint32_t>(), a->tris.as<int32_t>(),
                  a->refined.as<int32_t>(), a->occ_slot.as<int64_t>(), a->hkeys.as<unsigned long long>(),
                  a->hvals.as<long long>(), a->hmask, derr);
        amr_creators(st, 3 * R, a->occ_slot.as<int64_t>(), a->hvals.as<long long>(), a->cflag.as<uint32_t>(),
                     a->crank.as<uint32_t>());
        launch_scan_u32(st, a->crank.as<uint32_t>(), 3 * R, a->part.as<uint32_t>());
        int herr = 0;
        ACU(cudaMemcpyAsync(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost, st));
        int64_t C = 0;  // (scan_total synchronises the stream)
        if (int rc = scan_total(a, a->crank.as<uint32_t>(), a->cflag.as<uint32_t>(), 3 * R, &C)) return rc;
        if (herr) return afail(FSS_ERR_CAPACITY, "amr: parent-pair table full");
        if (n + C > a->max_points) return afail(FSS_ERR_CAPACITY, "amr: more points than the handle's max_count");
        amr_newpts(st, 3 * R, n, a->refined.as<int32_t>(), a->tris.as<int32_t>(), a->occ_slot.as<int64_t>(),
                   a->cflag.as<uint32_t>(), a->crank.as<uint32_t>(), a->hvals.as<long long>(),
                   a->state5.as<double>(), a->parent.as<int32_t>());
        amr_split(st, R, q0, q1, seq, a->refined.as<int32_t>(), a->occ_slot.as<int64_t>(), a->hvals.as<long long>(),
                  a->cflag.as<uint32_t>(), a->tarea.as<double>(), a->tris.as<int32_t>(), a->keys.as<uint64_t>(),
                  a->rec_v.as<uint32_t>() + nrec, a->rec_d.as<double>() + nrec, a->rec_k.as<uint8_t>() + nrec);
        ACU(cudaGetLastError());
        nrec += 6 * R;
        n += C;
        seq += uint64_t(R);
        q0 = q1;
        q1 += 3 * R;
    }
    if (nrec > 0) {
        ACU(a->sort_tmp.ensure(sizeof(uint32_t) * size_t(nrec)));
        ACU(a->sort_perm.ensure(sizeof(int32_t) * size_t(nrec)));
        ACU(a->sort_perm_tmp.ensure(sizeof(int32_t) * size_t(nrec)));
        ACU(a->sort_hist.ensure(sizeof(uint32_t) * size_t(sort_scratch_words(nrec))));
        launch_sort(st, nrec, bits_for(n), a->rec_v.as<uint32_t>(), a->sort_tmp.as<uint32_t>(),
                    a->sort_perm.as<int32_t>(), a->sort_perm_tmp.as<int32_t>(), a->sort_hist.as<uint32_t>());
        amr_areas(st, nrec, a->rec_v.as<uint32_t>(), a->sort_perm.as<int32_t>(), a->rec_d.as<double>(),
                  a->rec_k.as<uint8_t>(), a->area.as<double>());
        ACU(cudaGetLastError());
    }
    ACU(cudaStreamSynchronize(st));
    a->n = n;
    a->ntri = q1;
    a->seq = seq;
    a->adj_ok = false;
    return FSS_OK;
}


extern "C" {

int fss_amr_create(int64_t n, int64_t ntri, const int32_t* tris, const int32_t* parent_verts, int64_t max_count,
                   int64_t max_tris, int device, fss_amr** out) {
    if (!out) return afail(FSS_ERR_INVALID, "null argument");
    *out = nullptr;
    if (n < 3 || ntri < 1 || !tris) return afail(FSS_ERR_INVALID, "bad mesh");
    if (max_count < n || max_tris < ntri) return afail(FSS_ERR_INVALID, "capacities below the mesh size");
    if (max_count > (int64_t(1) << 30) || 3 * max_tris > (int64_t(1) << 31) - 1)
        return afail(FSS_ERR_INVALID, "capacities too large");
    for (int64_t j = 0; j < 3 * ntri; j++)
        if (tris[j] < 0 || tris[j] >= n) return afail(FSS_ERR_INVALID, "triangle vertex out of range");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return afail(FSS_ERR_UNSUPPORTED, "no CUDA device");
    }
    if (device < 0 || device >= ndev) return afail(FSS_ERR_INVALID, "bad device ordinal");
    ACU(cudaSetDevice(device));
    cudaDeviceProp prop;
    ACU(cudaGetDeviceProperties(&prop, device));
    if (prop.major < 10) return afail(FSS_ERR_UNSUPPORTED, "this build targets sm_100a (Blackwell B200)");
    std::unique_ptr<fss_amr> a(new fss_amr());
    a->dev = device;
    a->n = n;
    a->ntri = ntri;
    a->max_points = max_count;
    a->max_tris = max_tris;
    ACU(cudaStreamCreateWithFlags(&a->st, cudaStreamNonBlocking));
    ACU(a->state5.ensure(sizeof(double) * 5 * size_t(max_count)));
    ACU(a->area.ensure(sizeof(double) * size_t(max_count)));
    ACU(a->tris.ensure(sizeof(int32_t) * 3 * size_t(max_tris)));
    ACU(a->keys.ensure(sizeof(uint64_t) * 3 * size_t(max_tris)));
    ACU(a->parent.ensure(sizeof(int32_t) * 2 * size_t(max_count)));
    const int64_t hcap = pow2_at_least(2 * max_count);
    a->hmask = hcap - 1;
    ACU(a->hkeys.ensure(sizeof(unsigned long long) * size_t(hcap)));
    ACU(a->hvals.ensure(sizeof(long long) * size_t(hcap)));
    ACU(a->err.ensure(sizeof(int)));
    // per-pass scratch at its largest (a generation holds at most max_tris
    // triangles; refinements are bounded by the free triangle slots), so
    // that refining allocates nothing
    const size_t mt = size_t(max_tris), mref = size_t(std::max<int64_t>((max_tris - ntri) / 3, 1));
    ACU(a->flag.ensure(sizeof(uint32_t) * mt));
    ACU(a->rank.ensure(sizeof(uint32_t) * mt));
    ACU(a->tarea.ensure(sizeof(double) * mt));
    ACU(a->part.ensure(sizeof(uint32_t) * size_t(scan_part_words(3 * max_tris))));
    ACU(a->refined.ensure(sizeof(int32_t) * mref));
    ACU(a->occ_slot.ensure(sizeof(int64_t) * 3 * mref));
    ACU(a->cflag.ensure(sizeof(uint32_t) * 3 * mref));
    ACU(a->crank.ensure(sizeof(uint32_t) * 3 * mref));
    ACU(a->rec_v.ensure(sizeof(uint32_t) * 6 * mref));
    ACU(a->rec_d.ensure(sizeof(double) * 6 * mref));
    ACU(a->rec_k.ensure(sizeof(uint8_t) * 6 * mref));
    ACU(a->sort_tmp.ensure(sizeof(uint32_t) * 6 * mref));
    ACU(a->sort_perm.ensure(sizeof(int32_t) * 6 * mref));
    ACU(a->sort_perm_tmp.ensure(sizeof(int32_t) * 6 * mref));
    ACU(a->sort_hist.ensure(sizeof(uint32_t) * size_t(sort_scratch_words(int64_t(6 * mref)))));
    // initial lists in increasing triangle order: key = triangle index
    std::vector<uint64_t> keys(3 * size_t(ntri));
    for (int64_t j = 0; j < ntri; j++) keys[3 * j] = keys[3 * j + 1] = keys[3 * j + 2] = uint64_t(j);
    std::vector<int32_t> par(2 * size_t(n), 0);
    if (parent_verts) std::memcpy(par.data(), parent_verts, sizeof(int32_t) * 2 * n);
    cudaStream_t st = a->st;
    ACU(cudaMemcpyAsync(a->tris.p, tris, sizeof(int32_t) * 3 * ntri, cudaMemcpyHostToDevice, st));
    ACU(cudaMemcpyAsync(a->keys.p, keys.data(), sizeof(uint64_t) * keys.size(), cudaMemcpyHostToDevice, st));
    ACU(cudaMemsetAsync(a->parent.p, 0, sizeof(int32_t) * 2 * size_t(max_count), st));
    ACU(cudaMemcpyAsync(a->parent.p, par.data(), sizeof(int32_t) * par.size(), cudaMemcpyHostToDevice, st));
    ACU(cudaMemsetAsync(a->hkeys.p, 0xff, sizeof(unsigned long long) * size_t(hcap), st));
    ACU(cudaMemsetAsync(a->hvals.p, 0x7f, sizeof(long long) * size_t(hcap), st));
    ACU(cudaMemsetAsync(a->err.p, 0, sizeof(int), st));
    ACU(amr_seed_parents(st, n, a->parent.as<int32_t>(), a->hkeys.as<unsigned long long>(), a->hvals.as<long long>(),
                         a->hmask, a->err.as<int>()));
    int herr = 0;
    ACU(cudaMemcpyAsync(&herr, a->err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    ACU(cudaStreamSynchronize(st));
    if (herr) return afail(FSS_ERR_CAPACITY, "amr: parent-pair table full");
    *out = a.release();
    return FSS_OK;
}

void fss_amr_destroy(fss_amr* a) {
    if (!a) return;
    cudaSetDevice(a->dev);
    cudaStreamSynchronize(a->st);
    delete a;
}

int fss_amr_counts(const fss_amr* a, int64_t* point_count, int64_t* tri_count) {
    if (!a) return afail(FSS_ERR_INVALID, "null handle");
    if (point_count) *point_count = a->n;
    if (tri_count) *tri_count = a->ntri;
    return FSS_OK;
}

int fss_amr_refine(fss_amr* a, int64_t* point_count, double* state5, double* area, double vorticity_tol,
                   double circulation_tol) {
    if (!a || !point_count || !state5 || !area) return afail(FSS_ERR_INVALID, "null argument");
    if (a->broken) return afail(FSS_ERR_STATE, "amr handle unusable after a capacity error");
    if (*point_count != a->n) return afail(FSS_ERR_INVALID, "point_count differs from the mesh's");
    if (a->n >= a->max_points) return FSS_OK;  // config1.point_count >= config1.max_count: nothing
    ACU(cudaSetDevice(a->dev));
    const int64_t n0 = a->n;
    ACU(cudaMemcpyAsync(a->state5.p, state5, sizeof(double) * 5 * n0, cudaMemcpyHostToDevice, a->st));
    ACU(cudaMemcpyAsync(a->area.p, area, sizeof(double) * n0, cudaMemcpyHostToDevice, a->st));
    if (int rc = amr_refine_device(a, vorticity_tol, circulation_tol)) {
        a->broken = true;
        return rc;
    }
    const int64_t n1 = a->n;
    if (n1 > n0)
        ACU(cudaMemcpyAsync(state5 + 5 * n0, a->state5.as<double>() + 5 * n0, sizeof(double) * 5 * (n1 - n0),
                            cudaMemcpyDeviceToHost, a->st));
    ACU(cudaMemcpyAsync(area, a->area.p, sizeof(double) * n1, cudaMemcpyDeviceToHost, a->st));
    ACU(cudaStreamSynchronize(a->st));
    *point_count = n1;
    return FSS_OK;
}

int fss_amr_get_mesh(const fss_amr* a, int32_t* tris, uint64_t* corner_keys, int32_t* parent_verts) {
    if (!a) return afail(FSS_ERR_INVALID, "null handle");
    ACU(cudaSetDevice(a->dev));
    if (tris)
        ACU(cudaMemcpyAsync(tris, a->tris.p, sizeof(int32_t) * 3 * a->ntri, cudaMemcpyDeviceToHost, a->st));
    if (corner_keys)
        ACU(cudaMemcpyAsync(corner_keys, a->keys.p, sizeof(uint64_t) * 3 * a->ntri, cudaMemcpyDeviceToHost, a->st));
    if (parent_verts)
        ACU(cudaMemcpyAsync(parent_verts, a->parent.p, sizeof(int32_t) * 2 * a->n, cudaMemcpyDeviceToHost, a->st));
    ACU(cudaStreamSynchronize(a->st));
    return FSS_OK;
}

int fss_amr_remesh(fss_amr* a, const double* moved5, double* target5, double omega, int64_t* n_fallback,
                   int64_t* n_not_found) {
    if (!a || !moved5 || !target5) return afail(FSS_ERR_INVALID, "null argument");
    if (a->broken) return afail(FSS_ERR_STATE, "amr handle unusable after a capacity error");
    ACU(cudaSetDevice(a->dev));
    const int64_t n = a->n;
    cudaStream_t st = a->st;
    ACU(a->moved.ensure(sizeof(double) * 5 * size_t(n)));
    ACU(a->target.ensure(sizeof(double) * 5 * size_t(n)));
    if (!a->adj_ok) {
        ACU(a->off.ensure(sizeof(uint32_t) * size_t(a->max_points + 1)));
        ACU(a->adj.ensure(sizeof(int32_t) * 3 * size_t(a->max_tris)));
        bool valid = false;
        ACU(launch_remesh_adjacency(st, n, a->ntri, a->tris.as<int32_t>(), a->keys.as<uint64_t>(),
                                    a->off.as<uint32_t>(), a->adj.as<int32_t>(), a->rs, &valid));
        if (!valid) return afail(FSS_ERR_STATE, "amr mesh has a vertex out of range");
        a->adj_ok = true;
    }
    ACU(cudaMemcpyAsync(a->moved.p, moved5, sizeof(double) * 5 * n, cudaMemcpyHostToDevice, st));
    ACU(cudaMemcpyAsync(a->target.p, target5, sizeof(double) * 5 * n, cudaMemcpyHostToDevice, st));
    ACU(launch_remesh(st, n, a->moved.as<double>(), a->target.as<double>(), a->ntri, a->tris.as<int32_t>(),
                      a->off.as<uint32_t>(), a->adj.as<int32_t>(), omega, a->rs, n_fallback, n_not_found));
    ACU(cudaMemcpyAsync(target5, a->target.p, sizeof(double) * 5 * n, cudaMemcpyDeviceToHost, st));
    ACU(cudaStreamSynchronize(st));
    return FSS_OK;
}

}  // extern "C"
