"""Convert the HEALPix ring quadrature-weight FITS tables into one ``.npz`` file.

The weights themselves are data published with HEALPix and shipped by cuHPX
under the Apache-2.0 licence as ``cuhpx/data/weight_ring_nXXXXX.fits``
(read by ``cuhpx/sht_tools.py:34-44``).  Each file is a FITS BINTABLE with
``2*nside`` rows and three big-endian float64 columns (temperature, Q, U
weights); only column 0 is used.  This script decodes that table with a small
self-contained FITS reader (no astropy) and writes ``ring_weights.npz`` next to
itself, keyed ``n{nside}`` -> float64[2*nside].

Usage:  python cuhpx_b200/data/make_ring_weights.py <dir containing the .fits files>
"""

import os
import re
import sys

import numpy as np

BLOCK = 2880
CARD = 80


def _read_header(buf, off):
    """Parse one FITS header starting at byte ``off``; return (dict, data offset)."""
    cards = {}
    pos = off
    while True:
        if pos + CARD > len(buf):
            raise ValueError("FITS header has no END card")
        card = buf[pos : pos + CARD].decode("latin-1")
        pos += CARD
        key = card[:8].strip()
        if key == "END":
            break
        if card[8:10] == "= ":
            val = card[10:].split("/")[0].strip()
            if val.startswith("'"):
                val = val.strip("'").strip()
            cards[key] = val
    # header occupies whole 2880-byte blocks
    pos = off + ((pos - off + BLOCK - 1) // BLOCK) * BLOCK
    return cards, pos


def read_bintable_column0(path):
    """Return column 0 (a ``1D`` float64 column) of the first BINTABLE extension."""
    with open(path, "rb") as fh:
        buf = fh.read()
    prim, off = _read_header(buf, 0)
    naxis = int(prim.get("NAXIS", "0"))
    if naxis != 0:
        raise ValueError(f"{path}: primary HDU carries data; not a ring-weight table")
    ext, off = _read_header(buf, off)
    if ext.get("XTENSION") != "BINTABLE":
        raise ValueError(f"{path}: first extension is not a BINTABLE")
    row_bytes = int(ext["NAXIS1"])
    nrows = int(ext["NAXIS2"])
    tform1 = ext["TFORM1"].strip()
    m = re.fullmatch(r"(\d*)D", tform1)
    if m is None:
        raise ValueError(f"{path}: column 0 has TFORM {tform1}, expected a float64 column")
    repeat = int(m.group(1) or "1")
    raw = np.frombuffer(buf, dtype=np.uint8, count=row_bytes * nrows, offset=off)
    rows = raw.reshape(nrows, row_bytes)
    # a vector column ("1024D") stores several consecutive values per row; the
    # table is read row after row, as astropy's ``field(0).flatten()`` does
    col0 = rows[:, 0 : 8 * repeat].copy().view(">f8").reshape(nrows * repeat)
    return col0.astype(np.float64), int(ext.get("NSIDE", "0"))


def main(src_dir):
    out = {}
    for name in sorted(os.listdir(src_dir)):
        if not (name.startswith("weight_ring_n") and name.endswith(".fits")):
            continue
        w, nside = read_bintable_column0(os.path.join(src_dir, name))
        if nside == 0:
            nside = int(name[len("weight_ring_n") : -len(".fits")])
        if w.shape[0] != 2 * nside:
            raise ValueError(f"{name}: {w.shape[0]} rows, expected {2 * nside}")
        out[f"n{nside}"] = w
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ring_weights.npz")
    np.savez_compressed(dst, **out)
    print(f"wrote {dst}: {sorted(out, key=lambda k: int(k[1:]))}")


if __name__ == "__main__":
    # the FITS folder of a cuHPX checkout: first argument, or $CUHPX_REFERENCE/cuhpx/data
    src = sys.argv[1] if len(sys.argv) > 1 else None
    if src is None and os.environ.get("CUHPX_REFERENCE"):
        src = os.path.join(os.environ["CUHPX_REFERENCE"], "cuhpx", "data")
    if src is None:
        sys.exit("usage: make_ring_weights.py <cuHPX>/cuhpx/data  (or set CUHPX_REFERENCE)")
    main(src)
