"""Generate the golden vectors in ``tests/golden/*.npz`` from the cuHPX reference.

Runs the reference's own CPU transforms (``cuhpx.SHT`` / ``cuhpx.iSHT``,
cuhpx/hpx_sht.py:173-283, loaded by ``ref_loader.py``) on seeded inputs and
stores inputs and outputs.  Needs the cuHPX sources (first argument, or the
``CUHPX_REFERENCE`` environment variable); the fixtures it writes are
committed so that nothing else needs them.

Cases (each an ``.npz``):
  cfg1_n32     nside=32, L=M=65, one N(0,1) map (seed 0), 'ring' weights:
               SHT and iSHT in float64 and float32, and the round trip.
  small_nN     nside 2, 4, 8, 16 with the reference defaults L=4N-1, M=2N+1
               and with L=M=2N+1, float64 and float32.
  none_n8      nside=8 with quad_weights='none'.
  lm_n8        nside=8 with M > L (L=9, M=17) and M < L (L=17, M=5).
  sparse_n16   synthesis of a seeded sparse lower-triangular a_lm at L=M=33,
               then analysis (the round-trip recipe of the reference's
               tests/reproduce_cuhpx_sht_round_trip_error.py, own seed).
  grad_n8      autograd gradients of the reference CPU SHT/iSHT for the loss
               sum_lm |a_lm|^2/(l+1) and sum_p f_p^2 at nside=8, L=M=17.
"""

import os
import sys

import numpy as np
import torch

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from ref_loader import load_reference  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def run(hpx_sht, nside, L, M, f64, qw="ring"):
    sht = hpx_sht.SHT(nside, lmax=L, mmax=M, quad_weights=qw)
    isht = hpx_sht.iSHT(nside, lmax=L, mmax=M)
    x64 = torch.from_numpy(f64)
    a64 = sht(x64)
    a32 = sht(x64.to(torch.float32))
    b64 = isht(a64.clone())
    b32 = isht(a64.clone().to(torch.complex64))
    return dict(
        nside=nside,
        lmax=L,
        mmax=M,
        quad_weights=qw,
        f=f64,
        alm64=a64.numpy(),
        alm32=a32.numpy(),
        map64=b64.numpy(),
        map32=b32.numpy(),
    )


def main(ref_root=None):
    hpx_sht, _ = load_reference(ref_root)
    torch.set_num_threads(os.cpu_count() or 1)

    rng = np.random.default_rng(0)
    d = run(hpx_sht, 32, 65, 65, rng.standard_normal(12 * 32 * 32))
    np.savez_compressed(os.path.join(OUT, "cfg1_n32.npz"), **d)

    for nside in (2, 4, 8, 16):
        rng = np.random.default_rng(100 + nside)
        f = rng.standard_normal(12 * nside * nside)
        dd = run(hpx_sht, nside, 4 * nside - 1, 2 * nside + 1, f)
        de = run(hpx_sht, nside, 2 * nside + 1, 2 * nside + 1, f)
        np.savez_compressed(
            os.path.join(OUT, f"small_n{nside}.npz"),
            **{f"default_{k}": v for k, v in dd.items()},
            **{f"equal_{k}": v for k, v in de.items()},
        )

    rng = np.random.default_rng(8)
    f = rng.standard_normal(12 * 64)
    np.savez_compressed(os.path.join(OUT, "none_n8.npz"), **run(hpx_sht, 8, 17, 17, f, qw="none"))

    a = run(hpx_sht, 8, 9, 17, f)
    b = run(hpx_sht, 8, 17, 5, f)
    np.savez_compressed(
        os.path.join(OUT, "lm_n8.npz"), **{f"mgt_{k}": v for k, v in a.items()}, **{f"mlt_{k}": v for k, v in b.items()}
    )

    # sparse band-limited a_lm -> map -> a_lm
    nside, L = 16, 33
    rng = np.random.default_rng(42)
    alm = np.zeros((L, L), dtype=np.complex128)
    for _ in range(100):
        l = int(rng.integers(0, L - 1))
        m = int(rng.integers(0, l + 1))
        alm[l, m] = rng.random() + (1j * rng.random() if m > 0 else 0.0)
    sht = hpx_sht.SHT(nside, lmax=L, mmax=L)
    isht = hpx_sht.iSHT(nside, lmax=L, mmax=L)
    fmap = isht(torch.from_numpy(alm.copy()))
    back = sht(fmap)
    np.savez_compressed(
        os.path.join(OUT, "sparse_n16.npz"), nside=nside, lmax=L, mmax=L, alm=alm, map64=fmap.numpy(), alm_back64=back.numpy()
    )

    # autograd gradients of the reference CPU path
    nside, L = 8, 17
    rng = np.random.default_rng(7)
    f = torch.from_numpy(rng.standard_normal(12 * nside * nside)).requires_grad_(True)
    sht = hpx_sht.SHT(nside, lmax=L, mmax=L)
    isht = hpx_sht.iSHT(nside, lmax=L, mmax=L)
    wl = 1.0 / (torch.arange(L, dtype=torch.float64) + 1.0)
    a = sht(f)
    loss = (wl[:, None] * a.abs() ** 2).sum()
    loss.backward()
    alm_in = torch.from_numpy(
        rng.standard_normal((L, L)) + 1j * rng.standard_normal((L, L))
    ) * torch.tril(torch.ones(L, L, dtype=torch.float64))
    alm_in[:, 0] = alm_in[:, 0].real.to(torch.complex128)
    alm_req = alm_in.clone().requires_grad_(True)
    fm = isht(alm_req.clone())
    loss2 = (fm**2).sum()
    loss2.backward()
    np.savez_compressed(
        os.path.join(OUT, "grad_n8.npz"),
        nside=nside,
        lmax=L,
        mmax=L,
        f=f.detach().numpy(),
        loss=loss.item(),
        grad_f=f.grad.numpy(),
        alm=alm_in.numpy(),
        loss2=loss2.item(),
        grad_alm=alm_req.grad.numpy(),
    )
    print("golden fixtures written to", OUT)


if __name__ == "__main__":
    main(*(sys.argv[1:2]))
