"""Generate the golden fixtures in this folder from the reference's own FRCPU.

Runs only where the reference was compiled (``make -C oracle ref`` builds
``oracle/_ref/libfrcpu_ref.so`` from the reference sources).  Usage, from the repo root::

    python tests/golden/make_golden.py

Fixtures (numpy .npz, inputs and the reference's outputs):

* ``kat_<plane>_<type>_<interp>.npz`` -- the reference's own twelve unit cases
  (tests/operations/fourier_reconstruction/fr_tests.hpp:7-101, afr_common.hpp:316-427):
  a 5x6 projection (3x6 half-plane), a 7^3 volume, one axis-permutation rotation, FFT
  constant 1 (XY) or increasing 1, 2, 3, ... over the interleaved floats (YZ, XZ).
* ``rand_b<B>_<type>_<interp>.npz`` -- seeded synthetic jobs (umpalumpa_b200.synthetic).
* ``blob_table.npz`` -- the reference's 10,000-entry blob table (r 1.9, alpha 15, order 0).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from umpalumpa_b200 import synthetic  # noqa: E402

KAT_ROTATIONS = {
    "xy": np.eye(3, dtype=np.float32),
    "yz": np.array([[0, 0, 1], [0, 1, 0], [-1, 0, 0]], np.float32),
    "xz": np.array([[0, -1, 0], [0, 0, 1], [-1, 0, 0]], np.float32),
}
TYPES = {"fast": 0, "precise": 1}
INTERPS = {"dynamic": 0, "lookup": 1}


def kat_fft(plane: str) -> np.ndarray:
    n, y, x = 1, 6, 3
    if plane == "xy":
        f = np.ones(n * y * x * 2, np.float32)
    else:
        f = np.arange(1, n * y * x * 2 + 1, dtype=np.float32)
    return f.view(np.complex64).reshape(n, y, x)


def run_ref(fft, spaces, shape, type_, interp, table):
    vol = np.zeros(shape, np.complex64)
    w = np.zeros(shape, np.float32)
    oracle.fr_execute(vol, w, fft, spaces, table=table if interp else None, interpolation=interp,
                      type_=type_, impl="ref", threads=1)
    return vol, w


def main():
    if not oracle.ref_available():
        raise SystemExit("the reference FRCPU is not built; run `make -C oracle ref` first")
    table = oracle.fill_blob_table(impl="ref")
    np.savez_compressed(os.path.join(HERE, "blob_table.npz"), table=table)
    for plane, rot in KAT_ROTATIONS.items():
        for tname, t in TYPES.items():
            spaces = oracle.traverse_spaces(rot[None], 3, 6, 6, 6, use_fast=(t == 0), impl="ref")
            for iname, it in INTERPS.items():
                fft = kat_fft(plane)
                vol, w = run_ref(fft, spaces, (7, 7, 7), t, it, table)
                np.savez_compressed(os.path.join(HERE, f"kat_{plane}_{tname}_{iname}.npz"), fft=fft,
                                    spaces=spaces.view(np.uint8).reshape(-1, 112), volume=vol, weight=w)
    for box, n, seed, modes in ((16, 24, 7, [(t, i) for t in TYPES for i in INTERPS]),
                                (24, 40, 11, [("precise", "lookup"), ("precise", "dynamic")])):
        fft, rots = synthetic.make_job(box, n, seed=seed, snr=0.1)
        v = box + 1
        for tname, iname in modes:
            t, it = TYPES[tname], INTERPS[iname]
            spaces = oracle.traverse_spaces(rots, box // 2, box, box, box, use_fast=(t == 0), impl="ref")
            vol, w = run_ref(fft, spaces, (v, v, v), t, it, table)
            np.savez_compressed(os.path.join(HERE, f"rand_b{box}_{tname}_{iname}.npz"), fft=fft,
                                rotations=rots, spaces=spaces.view(np.uint8).reshape(-1, 112),
                                volume=vol, weight=w)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
