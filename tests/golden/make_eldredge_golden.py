"""Extract the golden force histories of the reference's pitch manoeuvre
(IBPM.jl ``benchmarks/eldredge``) into ``eldredge_pitch.json`` (moving grid:
``pitch_maneuver.jl`` wrote ``results/force_jl2.mat``) and
``eldredge_pitch_motion.json`` (moving body: ``pitch_maneuver_motion.jl`` wrote
``results/force_jl1.mat``; its run covered 10 000 of the 10 001 steps, the
last entry is zero and is dropped).

The .mat file is MATLAB v7.3 (an HDF5 file after a 512-byte header) holding
three float64 vectors of 10 001 entries, t, CL and CD (lab frame), stored
contiguously.  h5py is not available, so the vectors are read at their data
offset and identified by content: t is 0:1e-3:10, CD starts at the steady
flat-plate drag (≈ 0.394) and CL near zero.  Every 10th entry is kept.

Run from the repository root with the path of the reference tree:
    python tests/golden/make_eldredge_golden.py <IBPM.jl checkout>
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
FILES = (("force_jl2.mat", "eldredge_pitch.json", "pitch_maneuver.jl, MovingGrid", 10001),
         ("force_jl1.mat", "eldredge_pitch_motion.json", "pitch_maneuver_motion.jl, MotionFunction", 10000))
N = 10001       # entries stored per vector
OFFSET = 2560   # first byte of the contiguous data blocks
KEEP = 10


def extract(src, out, what, nkeep):
    raw = open(src, "rb").read()
    if not raw.startswith(b"MATLAB 7.3 MAT-file") or raw[512:520] != b"\x89HDF\r\n\x1a\n":
        sys.exit("not a MATLAB v7.3 (HDF5) file: %s" % src)
    blocks = np.frombuffer(raw, dtype="<f8", count=3 * N, offset=OFFSET).reshape(3, N)
    tref = np.arange(N) * 1e-3
    it = [k for k in range(3) if np.abs(blocks[k] - tref).max() < 1e-12]
    icd = [k for k in range(3) if abs(blocks[k][0] - 0.394) < 1e-3]
    icl = [k for k in range(3) if abs(blocks[k][0]) < 1e-5 and k not in it]
    if len(it) != 1 or len(icd) != 1 or len(icl) != 1 or len({it[0], icd[0], icl[0]}) != 3:
        sys.exit("could not identify t, CL and CD")
    t, cl, cd = blocks[it[0]][:nkeep], blocks[icl[0]][:nkeep], blocks[icd[0]][:nkeep]
    if not (np.all(np.isfinite(cl)) and np.all(np.isfinite(cd))) or cd[-1] == 0.0:
        sys.exit("non-finite or incomplete force history")
    sel = np.arange(0, nkeep, KEEP)
    doc = {
        "source": "IBPM.jl benchmarks/eldredge/results/%s (%s)" % (os.path.basename(src), what),
        "setup": {
            "boundary": [-1.5, 6.5, -2.0, 2.0], "h": 0.02, "mg": 5, "Re": 100.0,
            "plate": {"L": 1.0, "alpha": 0.0, "x0": 0.0, "y0": 0.0, "n": 51},
            "steady": {"dt": 1e-2, "steps": 10001, "freestream": [1.0, 0.0, 0.0]},
            "pitch": {"dt": 1e-3, "steps": nkeep, "a": 11.0, "t1234": [1.0, 3.0, 4.0, 6.0],
                      "alpha_max_deg": 45.0, "U": 1.0},
        },
        "steady_cd_published": {"julia": 0.39415052, "fortran": 0.39415060,
                                "where": "benchmarks/eldredge/README.md:25-26"},
        "step_stride": KEEP,
        "t": [float(v) for v in t[sel]],
        "CL_lab": [float(v) for v in cl[sel]],
        "CD_lab": [float(v) for v in cd[sel]],
    }
    with open(out, "w") as f:
        json.dump(doc, f, indent=0)
    print("wrote %s (%d samples)" % (out, sel.size))


def main(ref_root):
    results = os.path.join(ref_root, "benchmarks", "eldredge", "results")
    for name, out, what, nkeep in FILES:
        extract(os.path.join(results, name), os.path.join(HERE, out), what, nkeep)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_eldredge_golden.py <IBPM.jl checkout>")
    main(sys.argv[1])
