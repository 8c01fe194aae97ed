"""Golden vectors of the spin-1 (vector) transforms, from the reference itself.

Runs cuHPX's own ``VectorSHT`` / ``VectoriSHT`` (cuhpx/hpx_sht.py:286-444, with
``_precompute_dlegpoly`` of cuhpx/sht_tools.py:267-304) on seeded inputs.
Those classes call the CUDA ring-FFT module ``cuhpx_fft`` even on the CPU; its
``healpix_rfft_*`` / ``healpix_irfft_*`` are given here by the reference's own
CPU ring FFTs ``healpix_rfft_torch`` / ``healpix_irfft_torch``
(cuhpx/hpx_sht.py:37-76) applied map by map, which is what the batched CUDA
functions compute (src/harmonic_transform/hpx_fft.cpp:21-149).

    CUHPX_REFERENCE=/path/to/cuHPX python tests/golden/make_vector_golden.py
"""

import os
import sys

import numpy as np
import torch

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from ref_loader import load_reference  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def install_fft_shim(hpx_sht):
    fft = sys.modules["cuhpx_fft"]

    def per_map(fn, x, L, nside, lead_dims):
        lead = x.shape[:lead_dims]
        flat = x.reshape((-1,) + x.shape[lead_dims:])
        outs = [fn(flat[i].clone(), L, nside) for i in range(flat.shape[0])]
        out = torch.stack(outs)
        return out.reshape(lead + out.shape[1:])

    fft.healpix_rfft_class = lambda x, L, nside: hpx_sht.healpix_rfft_torch(x, L, nside)
    fft.healpix_rfft_batch = lambda x, L, nside: per_map(hpx_sht.healpix_rfft_torch, x, L, nside, x.dim() - 1)
    fft.healpix_irfft_class = lambda x, L, nside: hpx_sht.healpix_irfft_torch(x.clone(), L, nside)
    fft.healpix_irfft_batch = lambda x, L, nside: per_map(hpx_sht.healpix_irfft_torch, x, L, nside, x.dim() - 2)


def case(hpx_sht, nside, L, M, csphase, seed):
    rng = np.random.default_rng(seed)
    npix = 12 * nside * nside
    f = rng.standard_normal((2, npix))
    a = rng.standard_normal((2, L, M)) + 1j * rng.standard_normal((2, L, M))
    a = np.where(np.arange(M)[None, None, :] <= np.arange(L)[None, :, None], a, 0)
    a[..., 0] = a[..., 0].real
    a[:, 0, :] = 0  # degree 0 carries no vector field
    vs = hpx_sht.VectorSHT(nside, lmax=L, mmax=M, csphase=csphase)
    vi = hpx_sht.VectoriSHT(nside, lmax=L, mmax=M, csphase=csphase)
    alm = vs(torch.from_numpy(f)).numpy()
    vmap = vi(torch.from_numpy(a)).numpy()
    # autograd gradients of the reference: sum_lm |a_lm|^2 / (l+1) through
    # VectorSHT, and sum f^2 through VectoriSHT
    ft = torch.from_numpy(f).requires_grad_(True)
    wl = 1.0 / (torch.arange(L, dtype=torch.float64) + 1.0)[:, None]
    (vs(ft).abs() ** 2 * wl).sum().backward()
    at = torch.from_numpy(a).requires_grad_(True)
    (vi(at) ** 2).sum().backward()
    return dict(f=f, alm=alm, a=a, map=vmap, grad_f=ft.grad.numpy(), grad_a=at.grad.numpy())


def main(ref_root=None):
    hpx_sht, _ = load_reference(ref_root)
    install_fft_shim(hpx_sht)
    torch.set_num_threads(os.cpu_count() or 1)
    out = {}
    for name, (nside, L, M, cs, seed) in {
        "n8": (8, 17, 17, True, 21),
        "n8_nocs": (8, 17, 17, False, 22),
        "n4_mlt": (4, 9, 5, True, 23),
        "n4_mgt": (4, 7, 9, True, 24),
    }.items():
        d = case(hpx_sht, nside, L, M, cs, seed)
        for k, v in d.items():
            out[f"{name}_{k}"] = v
        out[f"{name}_cfg"] = np.array([nside, L, M, int(cs)])
        print(name, d["alm"].shape, d["map"].shape)
    np.savez_compressed(os.path.join(OUT, "vector_small.npz"), **out)


if __name__ == "__main__":
    main(*(sys.argv[1:2]))
