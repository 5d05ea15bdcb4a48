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
    print("wrote", sorted(f for f in os.listdir(HERE) if f.endswith(".npz")))


if __name__ == "__main__":
    main()
