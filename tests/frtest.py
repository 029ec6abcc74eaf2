"""Shared helpers for the Fourier-reconstruction tests."""
import glob
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")

# The reference's traverse-space known answers for a 5x6 projection (image size 3 x 6)
# inserted into a 7^3 volume (tests/operations/fourier_reconstruction/afr_common.hpp:136-254).
# Keys: (plane, type); values: ints (minY minX minZ maxY maxX maxZ), maxDistanceSqr, dir,
# unitNormal, topOrigin, bottomOrigin.  Weight 1, projectionIndex 0 in every case.
KAT_SPACES = {
    ("xy", "fast"): ((0, 3, 3, 6, 6, 3), 9.0, 0, (0, 0, 1), (6, 0, 3), (6, 0, 3)),
    ("xy", "precise"): ((0, 1, 1, 6, 6, 5), 24.0100002, 0, (0, 0, 1), (7.9, -1.9, 1.1), (7.9, -1.9, 4.9)),
    ("yz", "fast"): ((0, 3, 0, 6, 3, 3), 9.0, 2, (1, 0, 0), (3, 0, 0), (3, 0, 0)),
    ("yz", "precise"): ((0, 1, 0, 6, 5, 5), 24.0100002, 2, (1, 0, 0), (1.1, -1.9, -1.9), (4.9, -1.9, -1.9)),
    ("xz", "fast"): ((3, 0, 0, 3, 6, 3), 9.0, 1, (0, 1, 0), (6, 3, 0), (6, 3, 0)),
    ("xz", "precise"): ((1, 0, 0, 5, 6, 5), 24.0100002, 1, (0, 1, 0), (7.9, 1.1, -1.9), (7.9, 4.9, -1.9)),
}

KAT_ROTATIONS = {
    "xy": np.eye(3, dtype=np.float32),
    "yz": np.array([[0, 0, 1], [0, 1, 0], [-1, 0, 0]], np.float32),
    "xz": np.array([[0, -1, 0], [0, 0, 1], [-1, 0, 0]], np.float32),
}

TYPES = {"fast": 0, "precise": 1}
INTERPS = {"dynamic": 0, "lookup": 1}


def float_eq(a, b, ulps=4) -> bool:
    """gtest ASSERT_FLOAT_EQ: within 4 units in the last place."""
    a = np.float32(a)
    b = np.float32(b)
    if a == b:
        return True
    ia = np.array([a]).view(np.int32)[0]
    ib = np.array([b]).view(np.int32)[0]
    if (ia < 0) != (ib < 0):
        return False
    return abs(int(ia) - int(ib)) <= ulps


def check_kat_space(ts, plane: str, type_: str):
    """Compare one traverse space (structured record) with the reference's known answer."""
    ints, md, d, n, top, bot = KAT_SPACES[(plane, type_)]
    got = (int(ts["minY"]), int(ts["minX"]), int(ts["minZ"]), int(ts["maxY"]), int(ts["maxX"]), int(ts["maxZ"]))
    assert got == ints, (plane, type_, got, ints)
    assert float_eq(ts["maxDistanceSqr"], md), (ts["maxDistanceSqr"], md)
    assert int(ts["dir"]) == d
    for k in range(3):
        assert float_eq(ts["unitNormal"][k], n[k])
        assert float_eq(ts["topOrigin"][k], top[k]), (plane, type_, "top", ts["topOrigin"], top)
        assert float_eq(ts["bottomOrigin"][k], bot[k]), (plane, type_, "bottom", ts["bottomOrigin"], bot)
    assert float_eq(ts["weight"], 1.0)
    assert int(ts["projectionIndex"]) == 0


def check_structure(volume, weight, ts, max_distance):
    """The reference's structural check of one inserted projection (afr_common.hpp:256-314):
    zero outside the frequency sphere, behind the image or farther than max_distance from the
    plane; non-zero real, imaginary and weight everywhere else."""
    vz, vy, vx = weight.shape
    T = np.asarray(ts["transformInv"], np.float32)
    n = np.asarray(ts["unitNormal"], np.float32)
    md = np.float32(ts["maxDistanceSqr"])
    for z in range(vz):
        pz = np.float32(z - (vz - 1) // 2)
        for y in range(vy):
            py = np.float32(y - (vy - 1) // 2)
            for x in range(vx):
                px = np.float32(x - (vx - 1) // 2)
                v, w = volume[z, y, x], weight[z, y, x]
                zero = v.real == 0 and v.imag == 0 and w == 0
                nonzero = v.real != 0 and v.imag != 0 and w != 0
                if px * px + py * py + pz * pz > md:
                    assert zero, ("outside sphere", x, y, z, v, w)
                    continue
                ix = np.float32(T[0, 0] * px + T[0, 1] * py + T[0, 2] * pz)
                dist = abs(np.float32(n[0] * px + n[1] * py + n[2] * pz))
                if ix < -max_distance or dist > max_distance:
                    assert zero, ("off slab", x, y, z, v, w)
                else:
                    assert nonzero, ("on slab", x, y, z, v, w)


def load(name):
    d = np.load(os.path.join(GOLDEN, name))
    return {k: d[k] for k in d.files}


def golden_names(prefix):
    return sorted(os.path.basename(p) for p in glob.glob(os.path.join(GOLDEN, prefix + "*.npz")))


def parse_name(name):
    parts = name[:-4].split("_")
    return parts[1], parts[2], parts[3]


def rel_l2(a, b) -> float:
    a = np.asarray(a).astype(np.complex128 if np.iscomplexobj(a) else np.float64).ravel()
    b = np.asarray(b).astype(np.complex128 if np.iscomplexobj(b) else np.float64).ravel()
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / den) if den > 0 else float(np.linalg.norm(a - b))
