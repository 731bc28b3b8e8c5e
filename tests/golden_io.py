"""Loading of the golden fixtures in tests/golden (made by make_golden.py)."""
import glob
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def lab_cases():
    out = []
    for p in sorted(glob.glob(os.path.join(GOLDEN, "*.npz"))):
        z = np.load(p)
        meta = json.loads(str(z["meta"]))
        if meta["kind"] != "lab":
            continue
        bcl = {int(k): [tuple(e) for e in v] for k, v in meta["bcs"].items()}
        out.append(dict(name=os.path.basename(p)[:-4], comp=z["comp"], labs=z["labs"],
                        defined=z["defined"], nb=tuple(meta["nb"]), n=tuple(meta["n"]),
                        lo=tuple(meta["lo"]), hi=tuple(meta["hi"]),
                        tensorial=meta["tensorial"], blocks=meta["blocks"], bcs=bcl))
    return out


def c1_small():
    z = np.load(os.path.join(GOLDEN, "c1_small.npz"))
    meta = json.loads(str(z["meta"]))
    return dict(comp=z["comp"], lap=z["lap"], grad=z["grad"], nb=tuple(meta["nb"]),
                n=tuple(meta["n"]), h=meta["h"])
