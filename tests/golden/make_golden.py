"""Regenerate the golden fixtures from the reference itself.

Runs the reference's own functions (its headers compiled in place by
oracle/Makefile into oracle/_ref/libref.so) on small cases and stores their
outputs here, so that the oracle can be checked against the reference where
the reference's sources are absent:

    python tests/golden/make_golden.py     # needs oracle/_ref/libref.so
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402


def main():
    assert O.ref() is not None, "oracle/_ref/libref.so is not built (make -C oracle)"
    # icos_utils.h:15 icos_init, levels 0..3: vertices, faces, centres/radii
    verts, tv, ti = O.icos_init(3, use_ref=True)
    np.savez_compressed(os.path.join(HERE, "icos_l3.npz"), verts=verts, tri_verts=tv, tri_info=ti)
    # area_init + rossby_haurwitz_4 + rhs_func (direct) on the 162-particle grid
    s, a, tris = O.icos_state(2, use_ref=True)
    m = O.rhs_direct(s, a, use_ref=True)
    s1 = O.rk4_step(s, a, 0.01, use_ref=True)
    np.savez_compressed(os.path.join(HERE, "direct_l2.npz"), state=s, area=a, faces=tris, modify=m,
                        rk4_state=s1)
    # points_assign + tree_traverse on the 642-particle grid, 3 tree levels
    s3, a3, _ = O.icos_state(3, use_ref=True)
    loc, counts, pairs = O.ref_tree(3, 0.7, 10, s3)
    np.savez_compressed(os.path.join(HERE, "tree_l3.npz"), state=s3, loc=loc, counts=counts, pairs=pairs,
                        theta=0.7, many_count=10)
    # amr.h amr on the 162-point grid with a weakened Gaussian vortex
    # (vorticity_functions.h:26 gauss_vortex, zeta x 0.1), then
    # regrid_points2 with the vert_tris lists amr() left, on that mesh
    # rotated by 0.005 rad about z
    g, ga, gt = O.icos_state(2, use_ref=True)
    O.ref().ref_gauss_vortex(g.shape[0], g.reshape(-1), ga)
    g[:, 3] *= 0.1
    R = O.ref_amr(g, ga, gt, 10 * 4 ** 7 + 2)
    grid = R["state5"].copy()
    grid[:, :3] /= np.linalg.norm(grid[:, :3], axis=1, keepdims=True)
    c, sn = np.cos(0.005), np.sin(0.005)
    moved = grid.copy()
    moved[:, :3] = grid[:, :3] @ np.array([[c, -sn, 0], [sn, c, 0], [0, 0, 1]]).T
    out, rc = O.ref_remesh_lists(moved, grid, R["tris"], R["vert_tris"])
    assert rc == 0
    vt_off = np.concatenate([[0], np.cumsum([len(v) for v in R["vert_tris"]])]).astype(np.int32)
    np.savez_compressed(os.path.join(HERE, "amr_l2.npz"), state=g, area=ga, faces=gt, max_count=10 * 4 ** 7 + 2,
                        out_state=R["state5"], out_area=R["area"], out_tris=R["tris"], out_parent=R["parent"],
                        vt_off=vt_off, vt_adj=np.concatenate(R["vert_tris"]).astype(np.int32),
                        remesh_moved=moved, remesh_target=grid, remesh_out=out)
    print("wrote", sorted(f for f in os.listdir(HERE) if f.endswith(".npz")))


if __name__ == "__main__":
    main()
