"""Import the reference cuHPX CPU transforms (``SHT`` / ``iSHT``) from a source tree.

Only the fixture generator uses this, and only on a machine that has the
cuHPX sources.  The reference package does not import as shipped: its
``__init__`` pulls in ``torch_harmonics`` and two compiled extensions, and
``sht_tools`` needs astropy.  The CPU transforms need none of those, so this
loader builds a bare ``cuhpx`` package whose ``__path__`` is the reference's
own ``cuhpx/`` directory (so ``pkg_resources`` finds ``cuhpx/data``), stubs
the ``cuhpx_fft`` extension with an empty module, and stands in for
``astropy.io.fits.open`` with the FITS reader in ``make_ring_weights.py``.
"""

import importlib.util
import os
import sys
import types

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_REPO = os.path.dirname(os.path.dirname(_HERE))


def _fits_shim():
    sys.path.insert(0, os.path.join(_REPO, "cuhpx_b200", "data"))
    from make_ring_weights import read_bintable_column0

    class _Field:
        def __init__(self, col):
            self._col = col

        def field(self, i):
            if i != 0:
                raise KeyError(i)
            return self._col

    class _HDU:
        def __init__(self, col):
            self.data = _Field(col)

    class _HDUList(list):
        def __enter__(self):
            return self

        def __exit__(self, *a):
            return False

    def fits_open(path):
        col, _ = read_bintable_column0(path)
        return _HDUList([None, _HDU(col)])

    astropy = types.ModuleType("astropy")
    io = types.ModuleType("astropy.io")
    fits = types.ModuleType("astropy.io.fits")
    fits.open = fits_open
    io.fits = fits
    astropy.io = io
    sys.modules.setdefault("astropy", astropy)
    sys.modules.setdefault("astropy.io", io)
    sys.modules.setdefault("astropy.io.fits", fits)


def load_reference(ref_root=None):
    """Return the reference ``cuhpx.hpx_sht`` module (CPU classes usable).

    ``ref_root`` is a cuHPX checkout; by default the ``CUHPX_REFERENCE``
    environment variable names it.
    """
    ref_root = ref_root or os.environ.get("CUHPX_REFERENCE")
    if not ref_root:
        raise FileNotFoundError("no cuHPX checkout given (argument or CUHPX_REFERENCE)")
    pkg_dir = os.path.join(ref_root, "cuhpx")
    if not os.path.isdir(pkg_dir):
        raise FileNotFoundError(f"cuHPX sources not found at {pkg_dir}")
    _fits_shim()
    sys.modules.setdefault("cuhpx_fft", types.ModuleType("cuhpx_fft"))
    pkg = types.ModuleType("cuhpx")
    pkg.__path__ = [pkg_dir]
    pkg.__file__ = os.path.join(pkg_dir, "__init__.py")
    sys.modules["cuhpx"] = pkg
    mods = {}
    for name in ("sht_tools", "hpx_sht"):
        spec = importlib.util.spec_from_file_location(f"cuhpx.{name}", os.path.join(pkg_dir, f"{name}.py"))
        mod = importlib.util.module_from_spec(spec)
        sys.modules[f"cuhpx.{name}"] = mod
        spec.loader.exec_module(mod)
        setattr(pkg, name, mod)
        mods[name] = mod
    return mods["hpx_sht"], mods["sht_tools"]


if __name__ == "__main__":
    import torch

    hpx_sht, tools = load_reference()
    sht = hpx_sht.SHT(8, lmax=17, mmax=17)
    x = torch.randn(12 * 64, dtype=torch.float64)
    print(sht(x).shape, np.asarray(tools.healpix_weights(8, "ring")[1])[:3])
