"""The adjoint kernel behind peak_values: gradients of peak values and
|value|^2 with respect to data and template spectra, and through the torch
template generator to (alpha, t_c), against a torch.fft dense-correlation
gradient in FP64 and FP64 central finite differences (step 1e-6)."""
import numpy as np
import pytest

from apogee_b200 import synthetic

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    return torch


def dense_loss(D, H, idx, weights=None):
    """FP64 reference: sum over reported bins of |z|^2, or Re(conj(w) z), with
    z the dense torch.fft correlation gathered at the given lags."""
    torch = _torch()
    n = D.shape[-1]
    z = torch.fft.ifft(D[:, None, :] * torch.conj(H[None, :, :]), dim=-1) * n
    zb = torch.gather(z, 2, idx.clamp(min=0))
    mask = idx >= 0
    if weights is None:
        return ((zb.real ** 2 + zb.imag ** 2) * mask).sum()
    return ((torch.conj(weights) * zb).real * mask).sum()


def workload(n, nd, nt, seed):
    rng = np.random.default_rng(seed)
    H = synthetic.template_bank(n, nt, rng)
    D = synthetic.noise_spectra(n, nd, rng)
    for d in range(0, nd, 3):
        synthetic.inject(D, H, d, int(rng.integers(nt)), int(rng.integers(n)), 8.0)
    return D.astype(np.complex64), H


def reference_grads(D32, H32, idx, weights=None):
    torch = _torch()
    D = D32.detach().to(torch.complex128).requires_grad_(True)
    H = H32.detach().to(torch.complex128).requires_grad_(True)
    dense_loss(D, H, idx, weights).backward()
    return D.grad.resolve_conj(), H.grad.resolve_conj()


def assert_close(ours, ref, rel_l2=2e-5, rel_max=2e-4):
    """FP32 adjoint against the FP64 gradient: relative L2 error and largest
    elementwise error relative to the largest gradient component."""
    torch = _torch()
    ours = ours.to(torch.complex128)
    diff = ours - ref
    scale = ref.abs().max().item()
    assert scale > 0
    assert (diff.norm() / ref.norm()).item() <= rel_l2, (diff.norm() / ref.norm()).item()
    assert diff.abs().max().item() <= rel_max * scale, diff.abs().max().item() / scale


@pytest.mark.parametrize("n,nd,nt,binsize,thr", [
    (16384, 8, 256, 1024, 0.0),      # the differentiable-peaks workload
    (1024, 3, 40, 16, 0.0),          # many bins per pair
    (4096, 1, 7, 4096, 4.5),         # one bin, thresholded, split over templates
    (65536, 2, 3, 4096, 0.0),        # two-pass forward
])
def test_power_gradient_matches_dense_fp64(n, nd, nt, binsize, thr):
    torch = _torch()
    from apogee_b200.adjoint import peak_values
    Dn, Hn = workload(n, nd, nt, seed=n + nd)
    D = torch.from_numpy(Dn).cuda().requires_grad_(True)
    H = torch.from_numpy(Hn).cuda().requires_grad_(True)
    idx, val, power = peak_values(D, H, binsize, threshold=thr)
    power.sum().backward()
    if thr > 0:
        assert (idx < 0).any() and (idx >= 0).any()
    gD, gH = reference_grads(D, H, idx)
    assert_close(D.grad, gD)
    assert_close(H.grad, gH)


def test_value_gradient_and_forward_values():
    torch = _torch()
    import apogee_b200 as mf
    from apogee_b200.adjoint import peak_values
    n, nd, nt, binsize = 16384, 4, 32, 1024
    Dn, Hn = workload(n, nd, nt, seed=5)
    D = torch.from_numpy(Dn).cuda().requires_grad_(True)
    H = torch.from_numpy(Hn).cuda().requires_grad_(True)
    idx, val, power = peak_values(D, H, binsize)
    from oracle import oracle, parity
    bad = parity.compare(idx.cpu().numpy(), val.detach().cpu().numpy(),
                         oracle.correlate(Dn, Hn), binsize)
    assert not bad, bad[:3]
    f = mf.MatchedFilter(n, nd, nt)
    f.set_data(Dn)
    f.set_templates(Hn)
    ref = f.run(binsize=binsize)
    np.testing.assert_array_equal(idx.cpu().numpy(), ref["index"])
    np.testing.assert_array_equal(val.detach().cpu().numpy(), ref["value"])
    g = torch.Generator(device="cuda").manual_seed(1)
    w = torch.randn(val.shape, dtype=torch.complex64, device="cuda", generator=g)
    (torch.conj(w) * val).real.sum().backward()
    gD, gH = reference_grads(D, H, idx, w.to(torch.complex128))
    assert_close(D.grad, gD)
    assert_close(H.grad, gH)


def test_directional_finite_difference_fp64():
    torch = _torch()
    from apogee_b200.adjoint import peak_values
    n, nd, nt, binsize = 16384, 8, 256, 1024
    Dn, Hn = workload(n, nd, nt, seed=9)
    D = torch.from_numpy(Dn).cuda().requires_grad_(True)
    H = torch.from_numpy(Hn).cuda().requires_grad_(True)
    idx, val, power = peak_values(D, H, binsize)
    power.sum().backward()
    g = torch.Generator(device="cuda").manual_seed(2)
    VD = torch.randn(D.shape, dtype=torch.complex128, device="cuda", generator=g)
    VH = torch.randn(H.shape, dtype=torch.complex128, device="cuda", generator=g)
    D64, H64 = D.detach().to(torch.complex128), H.detach().to(torch.complex128)
    h = 1e-6
    with torch.no_grad():
        fd = (dense_loss(D64 + h * VD, H64 + h * VH, idx)
              - dense_loss(D64 - h * VD, H64 - h * VH, idx)).item() / (2 * h)
    an = ((torch.conj(D.grad.to(torch.complex128)) * VD).real.sum()
          + (torch.conj(H.grad.to(torch.complex128)) * VH).real.sum()).item()
    assert abs(fd - an) <= 1e-4 * abs(an), (fd, an)


def test_template_parameter_gradient():
    """d sum|peak|^2 / d(alpha, t_c) through the torch template generator and the
    adjoint, against FP64 central finite differences of the dense loss."""
    torch = _torch()
    from apogee_b200.adjoint import peak_values
    n, nd, nt, binsize = 16384, 8, 16, 1024
    rng = np.random.default_rng(11)
    alpha0 = rng.uniform(1e2, 1e4, size=nt)
    tc0 = rng.uniform(0, n, size=nt)
    Dn = synthetic.noise_spectra(n, nd, rng)
    H0 = synthetic.template_bank_torch(n, torch.tensor(alpha0), torch.tensor(tc0)).numpy()
    for d in range(nd):
        synthetic.inject(Dn, H0, d, d % nt, int(rng.integers(n)), 10.0)
    D = torch.from_numpy(Dn.astype(np.complex64)).cuda()
    alpha = torch.tensor(alpha0, device="cuda", requires_grad=True)
    tc = torch.tensor(tc0, device="cuda", requires_grad=True)
    H = synthetic.template_bank_torch(n, alpha, tc).to(torch.complex64)
    idx, val, power = peak_values(D, H, binsize)
    power.sum().backward()
    D64 = D.to(torch.complex128)

    def loss(a, t):
        with torch.no_grad():
            return dense_loss(D64, synthetic.template_bank_torch(n, a, t), idx).item()
    h = 1e-6
    a0, t0 = alpha.detach(), tc.detach()
    fd_a = np.empty(nt)
    fd_t = np.empty(nt)
    for i in range(nt):
        e = torch.zeros(nt, dtype=torch.float64, device="cuda")
        e[i] = h
        fd_a[i] = (loss(a0 + e, t0) - loss(a0 - e, t0)) / (2 * h)
        fd_t[i] = (loss(a0, t0 + e) - loss(a0, t0 - e)) / (2 * h)
    ga, gt = alpha.grad.cpu().numpy(), tc.grad.cpu().numpy()
    np.testing.assert_allclose(ga, fd_a, rtol=0, atol=1e-3 * np.abs(fd_a).max())
    np.testing.assert_allclose(gt, fd_t, rtol=0, atol=1e-3 * np.abs(fd_t).max())
