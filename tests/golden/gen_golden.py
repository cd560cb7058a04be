"""Generates the golden fixtures tests/golden/*.npz from the reference itself.

The outputs come from the reference's own lane_packing device code, compiled
unchanged into oracle/_ref/libcp_refcheck.so (make -C oracle ref), run on a GPU.
The inputs are seeded and saved beside the outputs.  Usage (on a GPU machine):
    python tests/golden/gen_golden.py [out_dir]
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import refcheck  # noqa: E402
from tests import boxgen  # noqa: E402

SIZES_COARSE = [64, 16, 16, 8]
SIZES_FINE = [512, 256, 256, 64]
FINE_WINDOWS = [(0.62, 0.6201), (0.9, 0.9001), (0.985, 0.98501)]


def family_fixture(fam: int) -> dict:
    dims = boxgen.DIMS[fam]
    out = {}
    lat_lo, lat_hi, specs = [], [], []
    idx = boxgen.lattice_indices(fam, SIZES_COARSE[:dims], 1500, seed=1000 + fam)
    lo, hi = refcheck.lattice_boxes(fam, boxgen.LAMBDA, SIZES_COARSE[:dims], idx)
    out["coarse_idx"] = idx
    out["coarse_lo"], out["coarse_hi"] = lo, hi
    parts = [(lo, hi), boxgen.sub_boxes(lo, hi, seed=2000 + fam), boxgen.point_boxes(lo[:, :500], hi[:, :500], 3000 + fam)]
    for j, w in enumerate(FINE_WINDOWS):
        fidx = boxgen.lattice_indices(fam, SIZES_FINE[:dims], 500, seed=4000 + 10 * fam + j)
        flo, fhi = refcheck.lattice_boxes(fam, w, SIZES_FINE[:dims], fidx)
        out[f"fine{j}_idx"] = fidx
        out[f"fine{j}_lo"], out[f"fine{j}_hi"] = flo, fhi
        parts.append((flo, fhi))
    blo = np.concatenate([p[0] for p in parts], axis=1)
    bhi = np.concatenate([p[1] for p in parts], axis=1)
    out["box_lo"], out["box_hi"] = blo, bhi
    out["box_bits"] = refcheck.eval_boxes(fam, blo, bhi)
    return out


def primitive_fixture() -> dict:
    from tests.test_parity_gpu import _prim_args

    out = {}
    for kind in range(6):
        args = _prim_args(kind, seed=50 + kind, n=2000)
        lo, hi, trap = refcheck.primitive(kind, args)
        out[f"k{kind}_args"], out[f"k{kind}_lo"], out[f"k{kind}_hi"], out[f"k{kind}_trap"] = args, lo, hi, trap
    rng = np.random.default_rng(60)
    x = np.concatenate([rng.uniform(-1, 1, 4000), rng.uniform(0.999, 1, 1000), [0.0, -0.0, 1.0, -1.0]])
    out["asin_x"] = x
    out["asin_rd"], out["asin_ru"] = refcheck.asin_pad(x)
    lam = np.linspace(0.5, 0.9900000000000001, 1001)
    out["single_lambda"] = lam
    out["single_out"] = refcheck.single_placement(lam)
    return out


def main():
    out_dir = sys.argv[1] if len(sys.argv) > 1 else os.path.join(ROOT, "tests", "golden")
    os.makedirs(out_dir, exist_ok=True)
    for fam in range(6):
        np.savez_compressed(os.path.join(out_dir, f"ref_{boxgen.FAMILY_NAMES[fam]}.npz"), **family_fixture(fam))
    np.savez_compressed(os.path.join(out_dir, "ref_primitives.npz"), **primitive_fixture())
    print("traps recorded by the reference checker:", refcheck.trap_count_reset())


if __name__ == "__main__":
    main()
