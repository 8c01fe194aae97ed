"""Golden vectors of the healpy a_lm index map, from the reference's own helpers.

cuHPX states the healpy packing in ``tests/reproduce_difference_between_healpy_cuhpx.py``
(``hp_getidx`` and ``flm_hp_to_2d``, lines 58-81).  That file imports healpy,
which is not installed here, so this script takes the two pure-Python functions
(and ``flm_shape``) out of it with ``ast`` and runs them as they are on a packed
vector whose entries are their own (complex) indices.  The output, committed as
``healpy_index_L8.npz`` and ``healpy_index_L13.npz``, pins the oracle's
restatement (``oracle/healpy_oracle.py``).

    CUHPX_REFERENCE=/path/to/cuHPX python tests/golden/make_healpy_golden.py
"""

import ast
import os
import sys

import numpy as np

OUT = os.path.dirname(os.path.abspath(__file__))
SRC = "tests/reproduce_difference_between_healpy_cuhpx.py"


def load_helpers(ref_root):
    path = os.path.join(ref_root, SRC)
    tree = ast.parse(open(path).read(), path)
    keep = [n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name in ("flm_shape", "hp_getidx", "flm_hp_to_2d")]
    mod = ast.Module(body=keep, type_ignores=[])
    ns = {"np": np}
    exec(compile(mod, path, "exec"), ns)
    return ns


def main(ref_root=None):
    ref_root = ref_root or os.environ.get("CUHPX_REFERENCE")
    if not ref_root:
        sys.exit("give the cuHPX checkout as the first argument or in CUHPX_REFERENCE")
    ns = load_helpers(ref_root)
    for L in (8, 13):
        n = L * (L + 1) // 2
        packed = np.arange(n) * (1.0 + 0.5j) + 0.25j  # every entry distinct, none real
        flm2d = ns["flm_hp_to_2d"](packed, L)
        idx = np.array([[ns["hp_getidx"](L, el, m) for m in range(L)] for el in range(L)])
        np.savez_compressed(os.path.join(OUT, f"healpy_index_L{L}.npz"), packed=packed, flm2d=flm2d, hp_getidx=idx)
        print("wrote", f"healpy_index_L{L}.npz", flm2d.shape)


if __name__ == "__main__":
    main(*(sys.argv[1:2]))
