"""Loader of the golden fixtures (tests/golden/golden.npz, made by
tests/golden/make_golden.py from the reference plugin's own outputs)."""
import json
import os

import numpy as np

PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden.npz")


def load():
    z = np.load(PATH)
    meta = json.loads(bytes(z["meta"]).decode())
    clips = {}
    for name in meta["clips"]:
        clips[name] = [z[f"{name}_in{i}"] for i in range(3)]
    cases = []
    for c in meta["cases"]:
        ins = clips[c["clip"]]
        outs = [(ins[i].astype(np.int32) + z[f"{c['name']}_diff{i}"]).astype(ins[i].dtype) for i in range(3)]
        cases.append((c["name"], clips[c["clip"]], c["bits"], c["params"], outs))
    return cases
