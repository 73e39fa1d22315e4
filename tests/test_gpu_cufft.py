"""Cross-check of the hand-written FFT convolution against cuFFT.

The open-boundary solve (openBC3D, Field.f90:239-331) convolves the charge
with the integrated Green function on the doubled grid.  Here the library's
potential for the charge it deposited is compared with the same convolution
done by torch.fft (cuFFT) in FP64 on the GPU, on configs[1]'s 64x64x128
grid: relative L2 <= 1e-12 in the plain FP64 form, <= 1e-5 in the
FP32-convolution form.  The Green function comes from the oracle's
greenf1tIntnew restatement; its even mirror makes the spectrum real, so the
forward sign convention does not matter (FFT.f90:26-250 fixes only signs and
the 1/(n1 n2 n3) scale).
"""
import numpy as np
import pytest

from conftest import load_impz, load_oracle

pytestmark = pytest.mark.gpu

impz = load_impz()
orc = load_oracle()
from impz_b200 import beams  # noqa: E402


def cufft_potential(rho, grid, msize):
    import torch
    nx, ny, nz = grid
    grn = np.zeros((nx + 1) * (ny + 1) * (nz + 1))
    orc.lib().orc_igf(nx, ny, nz, msize[0], msize[1], msize[2], orc.dp(grn))
    g = torch.from_numpy(grn.reshape(nz + 1, ny + 1, nx + 1)).cuda()
    ii = torch.arange(2 * nx, device="cuda")
    jj = torch.arange(2 * ny, device="cuda")
    kk = torch.arange(2 * nz, device="cuda")
    ii = torch.where(ii <= nx, ii, 2 * nx - ii)
    jj = torch.where(jj <= ny, jj, 2 * ny - jj)
    kk = torch.where(kk <= nz, kk, 2 * nz - kk)
    gfull = g[kk][:, jj][:, :, ii]
    r = torch.zeros((2 * nz, 2 * ny, 2 * nx), dtype=torch.float64, device="cuda")
    r[:nz, :ny, :nx] = torch.from_numpy(rho.reshape(nz, ny, nx)).cuda()
    phi = torch.fft.irfftn(torch.fft.rfftn(r) * torch.fft.rfftn(gfull), s=r.shape)
    return phi[:nz, :ny, :nx].reshape(-1).cpu().numpy()


@pytest.mark.parametrize("form,tol", [(impz.FORM_FP64, 1e-12), (impz.FORM_FP32CONV, 1e-5)])
def test_convolution_equals_cufft(form, tol):
    cfg = beams.fodo_4e6(n=400_000, seed=beams.SEED0 + 41)
    b = impz.Bunch(cfg["pts"], cfg["current"], cfg["mass"], cfg["charge"], cfg["freq"],
                   cfg["refptcl"], cfg["grid"], form=form, track_ids=False)
    try:
        _, _, _, msize = b.sc_prepare(1.0, 1.0)
        rho, _ = b.deposit(want_counts=False)
        phi = b.poisson()
    finally:
        b.close()
    want = cufft_potential(rho, cfg["grid"], msize)
    err = float(np.linalg.norm(phi - want) / np.linalg.norm(want))
    print("form %d: potential vs cuFFT, relative L2 %.3e" % (form, err))
    assert err <= tol
