"""Extract mhs's image-family records into ``oracle/image_table.npz``.

Test infrastructure: the oracle reads its image coefficients from this file,
taken straight from mhs's generated table (mhs/kernels/_image_table.py), so
it shares no generated data with the CUDA library.  Run where the reference
tree exists, with its path as the argument or its ``src/`` directory in
``MHS_REFERENCE_SRC``::

    python oracle/make_table.py [path to mhs/kernels/_image_table.py]
"""
from __future__ import annotations

import ast
import os
import pathlib
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent


def main(src: str) -> None:
    tree = ast.parse(pathlib.Path(src).read_text())
    tab = {}
    for node in tree.body:
        if isinstance(node, ast.Assign) and len(node.targets) == 1:
            name = getattr(node.targets[0], "id", None)
            if name and name.endswith("RECORDS"):
                tab[name] = ast.literal_eval(node.value)
    out = {}
    for name, nix, nexp in (("DG_RECORDS", 3, 4), ("DDG_RECORDS", 4, 4),
                            ("Q_DG_RECORDS", 3, 5), ("Q_DDG_RECORDS", 4, 5)):
        recs = tab[name]
        idx = np.array([r[:nix] for r in recs], dtype=np.int64)
        exp = np.array([r[nix:nix + nexp] for r in recs], dtype=np.int64)
        # coefficient terms (record, pz, pnu, num, den), flattened
        terms = np.array([(i, t[0], t[1], t[2], t[3]) for i, r in enumerate(recs)
                          for t in r[nix + nexp]], dtype=np.int64)
        key = name.lower().replace("_records", "")
        out[f"{key}_idx"] = idx
        out[f"{key}_exp"] = exp
        out[f"{key}_terms"] = terms
    np.savez_compressed(HERE / "image_table.npz", **out)
    print("wrote", HERE / "image_table.npz", {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    if len(sys.argv) > 1:
        main(sys.argv[1])
    elif os.environ.get("MHS_REFERENCE_SRC"):
        main(os.path.join(os.environ["MHS_REFERENCE_SRC"], "mhs", "kernels", "_image_table.py"))
    else:
        sys.exit("usage: make_table.py <mhs/kernels/_image_table.py> "
                 "(or set MHS_REFERENCE_SRC to the reference's src/ directory)")
