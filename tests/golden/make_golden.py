"""Generates the golden fixtures in this directory from the reference.

Run from the repository root after `make -C oracle` (needs oracle/_ref/libref.so,
the reference rezucch1/nbody-FMM compiled from its own sources):

    python tests/golden/make_golden.py

Fixtures (inputs stored beside outputs, so tests never regenerate inputs):
  tree15.json     the reference's tests/test_tree.cpp case: 15 particles from
                  glibc srand(42)/rand() in [-100,100]^3, threshold 20, with the
                  leaf membership the reference produces; it is checked here
                  against the membership that test asserts (test_tree.cpp:63-99).
  ref_trees.npz   Tree::init_tree output (depth, leaves, membership, lists) for
                  seeded 2D/3D uniform, Plummer and clumped sets.
  ref_fmm2d.npz   FMM::update accelerations/G in 2D (uniform disk, where the
                  reference is accurate) at p = 2, 8, 15.
  ref_near3d.npz  FMM::update in 3D at L = 0: the far field's gradient is then
                  zero (local_set3D.cpp:88), leaving exactly the near-field
                  P2P sums of leaf.cpp:118-142.
  ref_harm.npz    PowerSet<3> and Irregular values, and MultipoleSet<3> P2M moments.
  ref_naive.npz   NaiveUpdate accelerations/G (2D and 3D) and 10 SyplecticEuler
                  steps with NaiveUpdate.
  ref_se.npz      SyplecticEuler trajectories with forces large enough to
                  move the state: 10 steps with NaiveUpdate (3D, 300 particles
                  of mass 1e8) and 10 steps with the 2D FMM (uniform disk,
                  1000 particles of mass 1e7, p = 12, threshold 16, where the
                  reference's 2D FMM is accurate).
  ref_tree_c2.json  Tree::init_tree on the 2^20 Plummer sphere (seed 2,
                  threshold 64; depth 10, the reference's 32-bit key limit):
                  depth, level sizes and SHA-256 digests of the leaf keys,
                  leaf starts and membership (the arrays are 17 MB; about a
                  minute of the reference's CPU).

    python tests/golden/make_golden.py [fixture ...]   (default: all)
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "nbody-fmm_b200"))
from oracle import RAND_MAX, RefLib, glibc_rand_sequence  # noqa: E402
from fmmgpu import workloads  # noqa: E402

# Leaf membership asserted by the reference's tests/test_tree.cpp:63-99.
TEST_TREE_EXPECTED = {0: [1, 4, 7, 14], 1: [11], 3: [2, 13], 4: [0, 3], 5: [5], 6: [10, 12], 7: [6, 8, 9]}


def tree15(R):
    r = glibc_rand_sequence(42, 45)
    pos = ((r * 2.0 * 100.0) / RAND_MAX - 100.0).reshape(15, 3)
    t = R.tree(pos, 20)
    leaves = {int(k): t["perm"][s:e].tolist() for k, s, e in zip(t["leaf_keys"], t["leaf_start"][:-1], t["leaf_start"][1:])}
    assert t["depth"] == 1, t["depth"]
    assert leaves == TEST_TREE_EXPECTED, leaves
    return {"threshold": 20, "depth": 1, "positions_hex": [[float(v).hex() for v in row] for row in pos],
            "leaves": {str(k): v for k, v in leaves.items()}}


TREE_CASES = [
    ("u3_500_16", lambda: workloads.uniform_cube(500, seed=1)[0], 16),
    ("u3_3000_20", lambda: workloads.uniform_cube(3000, seed=7)[0], 20),
    ("pl3_20000_64", lambda: workloads.plummer(20000, seed=2)[0], 64),
    ("pl3_4000_8", lambda: workloads.plummer(4000, seed=9)[0], 8),
    ("u2_2000_16", lambda: workloads.uniform_cube(2000, seed=3, dim=2)[0], 16),
    ("c2_5000_32", lambda: workloads.disk_clumps_2d(5000, seed=3)[0], 32),
]


def tree_digests(depth, leaf_keys, leaf_start, perm):
    """SHA-256 of the leaf arrays as little-endian uint64 / int64."""
    return {"leaf_keys": hashlib.sha256(np.asarray(leaf_keys, "<u8").tobytes()).hexdigest(),
            "leaf_start": hashlib.sha256(np.asarray(leaf_start, "<i8").tobytes()).hexdigest(),
            "perm": hashlib.sha256(np.asarray(perm, "<i8").tobytes()).hexdigest()}


def tree_c2(R):
    from oracle import _d, _i64, _p, _u64

    pos, _ = workloads.plummer(1 << 20, seed=2)
    R.L.ref_set_params(2, 64)
    D = R.L.ref_tree_build(3, len(pos), _p(pos, _d), _p(np.ones(len(pos)), _d))
    sizes = [int(R.L.ref_tree_level_size(d)) for d in range(D + 1)]
    keys = np.zeros(sizes[D], np.uint64)
    start = np.zeros(sizes[D] + 1, np.int64)
    perm = np.zeros(len(pos), np.int64)
    R.L.ref_tree_leaves(_p(keys, _u64), _p(start, _i64), _p(perm, _i64))
    R.L.ref_tree_free()
    out = {"workload": "plummer(1 << 20, seed=2)", "threshold": 64, "depth": int(D), "level_sizes": sizes,
           "sha256": tree_digests(D, keys, start, perm)}
    with open(os.path.join(HERE, "ref_tree_c2.json"), "w") as f:
        json.dump(out, f, indent=1)


def se_trajectories(R):
    out = {"G": np.array(R.G)}
    pos, _ = workloads.uniform_cube(300, seed=40)
    m = np.full(300, 1e8)
    vel = np.random.default_rng(41).normal(size=pos.shape) * 0.01
    x, v = R.se_steps(pos, vel, m, 1e-3, 10, use_fmm=False)
    out.update({"naive3/pos": pos, "naive3/vel": vel, "naive3/mass": m, "naive3/x": x, "naive3/v": v})
    pos, _ = workloads.uniform_disk_2d(1000, seed=42)
    m = np.full(1000, 1e7)
    vel = np.random.default_rng(43).normal(size=pos.shape) * 0.01
    x, v = R.se_steps(pos, vel, m, 1e-3, 10, use_fmm=True, p=12, threshold=16)
    out.update({"fmm2/pos": pos, "fmm2/vel": vel, "fmm2/mass": m, "fmm2/x": x, "fmm2/v": v,
                "fmm2/p": np.array(12), "fmm2/T": np.array(16)})
    np.savez_compressed(os.path.join(HERE, "ref_se.npz"), **out)


def main():
    R = RefLib()
    which = set(sys.argv[1:]) or {"base", "se", "tree_c2"}
    if "se" in which:
        se_trajectories(R)
    if "tree_c2" in which:
        tree_c2(R)
    if "base" not in which:
        print("fixtures written to", HERE)
        return
    with open(os.path.join(HERE, "tree15.json"), "w") as f:
        json.dump(tree15(R), f, indent=1)

    out = {}
    for name, gen, T in TREE_CASES:
        pos = gen()
        t = R.tree(pos, T)
        out[f"{name}/pos"] = pos
        out[f"{name}/T"] = np.array(T)
        out[f"{name}/depth"] = np.array(t["depth"])
        out[f"{name}/leaf_keys"] = t["leaf_keys"]
        out[f"{name}/leaf_start"] = t["leaf_start"]
        out[f"{name}/perm"] = t["perm"]
        for d in range(t["depth"] + 1):
            out[f"{name}/level{d}"] = t["level_keys"][d]
            if len(pos) > 5000:
                continue  # membership only for the large case (keeps the fixture small)
            for kind in (0, 1):
                tk, sk = t["pairs"][d][kind]
                o = np.lexsort((sk, tk))
                out[f"{name}/pairs{d}_{kind}"] = np.stack([tk[o], sk[o]]) if len(tk) else np.zeros((2, 0), np.uint64)
    np.savez_compressed(os.path.join(HERE, "ref_trees.npz"), **out)

    pos, m = workloads.uniform_disk_2d(1000, seed=11)
    f2 = {"pos": pos, "mass": m}
    for p in (2, 8, 15):
        f2[f"p{p}"] = R.fmm(pos, m, p, 16)
    np.savez_compressed(os.path.join(HERE, "ref_fmm2d.npz"), **f2)

    pos, m = workloads.uniform_cube(2000, seed=12)
    m = np.random.default_rng(12).random(2000) + 0.5
    np.savez_compressed(os.path.join(HERE, "ref_near3d.npz"), pos=pos, mass=m, T=np.array(16),
                        grad=R.fmm(pos, m, 0, 16))

    rng = np.random.default_rng(13)
    vecs = rng.normal(size=(8, 3))
    P = 12
    reg = np.stack([R.regular_3d(P, v) for v in vecs])
    irr = np.stack([R.irregular_3d(P, v) for v in vecs])
    ppos = rng.normal(size=(30, 3)) * 0.3
    pm = rng.random(30) + 0.1
    pc = np.array([0.05, -0.02, 0.01])
    p2m = R.p2m_3d(8, ppos, pm, pc)
    np.savez_compressed(os.path.join(HERE, "ref_harm.npz"), p=np.array(P), vecs=vecs, regular=reg, irregular=irr,
                        p2m_pos=ppos, p2m_mass=pm, p2m_centre=pc, p2m=p2m)

    nv = {}
    for dim in (2, 3):
        pos, m = workloads.uniform_cube(300, seed=20 + dim, dim=dim)
        vel = np.random.default_rng(30 + dim).normal(size=pos.shape) * 0.01
        nv[f"d{dim}/pos"] = pos
        nv[f"d{dim}/mass"] = m
        nv[f"d{dim}/vel"] = vel
        nv[f"d{dim}/grad"] = R.naive(pos, m)
        x, v = R.se_steps(pos, vel, m, 1e-3, 10, use_fmm=False)
        nv[f"d{dim}/se_x"] = x
        nv[f"d{dim}/se_v"] = v
    nv["G"] = np.array(R.G)
    np.savez_compressed(os.path.join(HERE, "ref_naive.npz"), **nv)
    print("fixtures written to", HERE)


if __name__ == "__main__":
    main()
