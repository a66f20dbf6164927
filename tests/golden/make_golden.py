"""Writes tests/golden/golden.json.

Contents:
  * published_linear_modes_L1 -- the L1 error table of the damped EMHD
    linear mode as published in the reference
    (src/problem/linear_modes/Linear modes.ipynb, cell 1);
  * cases -- oracle snapshots (sum of each primitive over the interior and
    one probe zone) after a few steps of each workload at 16^2, so later
    changes of the oracle are caught.

Run from the repository root:  python tests/golden/make_golden.py
"""
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from grim_b200 import config as C  # noqa: E402
from grim_b200 import problems as PR  # noqa: E402
from oracle import oracle as O  # noqa: E402

PUBLISHED = {
    "N": [32, 64, 128, 256, 512],
    "errors": {
        "rho": [3.988654e-12, 4.969112e-13, 5.100655e-14, 9.139936e-15, 1.210917e-15],
        "u": [1.169794e-11, 1.228705e-12, 1.224386e-13, 1.150570e-14, 1.428690e-15],
        "u1": [2.550613e-13, 4.841199e-14, 6.637352e-15, 5.871516e-16, 6.168086e-17],
        "u2": [1.426849e-12, 1.326205e-13, 9.958794e-15, 1.233547e-15, 2.263401e-16],
        "q": [6.370257e-12, 5.447082e-13, 4.694195e-14, 4.554252e-15, 7.538579e-16],
        "dP": [4.509557e-12, 4.659176e-13, 4.400123e-14, 4.295960e-15, 5.914910e-16],
        "B1": [4.857199e-13, 7.734114e-14, 8.072464e-15, 5.271674e-16, 9.312974e-17],
        "B2": [3.446792e-13, 4.281455e-14, 4.445065e-15, 3.543071e-16, 5.441856e-17],
    },
    "source": "src/problem/linear_modes/Linear modes.ipynb cell 1",
}

CASES = {
    "fast_mode_16": dict(config=PR.fast_mode_config(N=16), prims="fast_mode_prims", steps=3),
    "linear_modes_16": dict(config=PR.linear_modes_config(N=16), prims="linear_modes_prims",
                            prims_kw=dict(amplitude=1e-4), steps=3),
    "orszag_tang_16": dict(config=PR.orszag_tang_config(N=16), prims="orszag_tang_prims", steps=2),
    "emhd_stratified_16": dict(config=PR.emhd_stratified_config(N=16), prims="emhd_stratified_prims", steps=2),
}


def main():
    out = {"published_linear_modes_L1": PUBLISHED, "cases": {}}
    for name, case in CASES.items():
        cfg = case["config"]
        P = getattr(PR, case["prims"])(cfg, **case.get("prims_kw", {}))
        o = O.Oracle(cfg)
        o.set_prims(P)
        o.time_step(case["steps"])
        Q = o.get_prims()
        s3, s2, s1 = C.interior_slices(cfg)
        probe_index = [0, 7, 9] if cfg["dim"] == 2 else [5, 7, 9]
        out["cases"][name] = dict(
            config={k: v for k, v in cfg.items()}, prims=case["prims"], prims_kw=case.get("prims_kw", {}),
            steps=case["steps"], time=o.time,
            var_sums=[float(x) for x in np.sum(Q[:, s3, s2, s1], axis=(1, 2, 3))],
            probe_index=probe_index, probe=[float(x) for x in Q[(slice(None),) + tuple(probe_index)]])
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print("wrote", path)


if __name__ == "__main__":
    main()
