"""CPU checks of the adjoint's checkers: the torch template generator against
the numpy one, and the closed-form adjoint the kernel evaluates against a
torch.fft dense-correlation gradient and FP64 central finite differences."""
import numpy as np
import torch

from apogee_b200 import synthetic


def dense_loss(D, H, idx, weights=None):
    """Sum over reported bins of |z|^2 (or Re(conj(w) z)), z from the dense
    torch.fft correlation z[k] = n * ifft(D conj(H))[k], gathered at idx."""
    n = D.shape[-1]
    z = torch.fft.ifft(D[:, None, :] * torch.conj(H[None, :, :]), dim=-1) * n
    zb = torch.gather(z, 2, idx.clamp(min=0))
    mask = idx >= 0
    if weights is None:
        return ((zb.real ** 2 + zb.imag ** 2) * mask).sum()
    return ((torch.conj(weights) * zb).real * mask).sum()


def closed_form(D, H, idx, gz):
    """grad_D[d,f] = sum_tb g H[t,f] W^-fk ; grad_H[t,f] = sum_db conj(g) D[d,f] W^+fk."""
    n = D.shape[1]
    f = np.arange(n)
    gD = np.zeros_like(D)
    gH = np.zeros_like(H)
    for d in range(D.shape[0]):
        for t in range(H.shape[0]):
            for b in range(idx.shape[2]):
                k = idx[d, t, b]
                if k < 0:
                    continue
                w = np.exp(2j * np.pi * f * k / n)
                g = gz[d, t, b]
                gD[d] += g * H[t] * np.conj(w)
                gH[t] += np.conj(g) * D[d] * w
    return gD, gH


def test_torch_generator_matches_numpy():
    n, nt = 1024, 5
    rng = np.random.default_rng(7)
    H = synthetic.template_bank(n, nt, np.random.default_rng(7)).astype(np.complex128)
    # the numpy bank draws alpha, then t_c, from the same seed
    alpha = rng.uniform(1e2, 1e4, size=nt)
    tc = rng.uniform(0, n, size=nt)
    Ht = synthetic.template_bank_torch(n, torch.tensor(alpha), torch.tensor(tc)).numpy()
    np.testing.assert_allclose(Ht, H, atol=2e-7)
    assert abs(np.linalg.norm(Ht[0]) - 1.0) < 1e-12
    np.testing.assert_allclose(Ht[:, n - 25], np.conj(Ht[:, 25]), atol=1e-15)


def test_closed_form_matches_dense_gradient_and_fd():
    n, nd, nt, nb = 128, 2, 3, 4
    rng = np.random.default_rng(3)
    D = rng.standard_normal((nd, n)) + 1j * rng.standard_normal((nd, n))
    H = rng.standard_normal((nt, n)) + 1j * rng.standard_normal((nt, n))
    idx = rng.integers(0, n, size=(nd, nt, nb))
    idx[0, 1, 2] = -1
    w = rng.standard_normal((nd, nt, nb)) + 1j * rng.standard_normal((nd, nt, nb))
    for weights in (None, w):
        Dt = torch.tensor(D, requires_grad=True)
        Ht = torch.tensor(H, requires_grad=True)
        it = torch.tensor(idx)
        wt = None if weights is None else torch.tensor(weights)
        dense_loss(Dt, Ht, it, wt).backward()
        if weights is None:
            z = np.fft.ifft(D[:, None, :] * np.conj(H[None]), axis=-1) * n
            gz = 2 * np.take_along_axis(z, np.maximum(idx, 0), axis=2)
        else:
            gz = weights
        gD, gH = closed_form(D, H, idx, gz)
        np.testing.assert_allclose(gD, Dt.grad.resolve_conj().numpy(), rtol=1e-10, atol=1e-9)
        np.testing.assert_allclose(gH, Ht.grad.resolve_conj().numpy(), rtol=1e-10, atol=1e-9)
        # FP64 central finite difference along a random direction, step 1e-6
        VD = rng.standard_normal((nd, n)) + 1j * rng.standard_normal((nd, n))
        VH = rng.standard_normal((nt, n)) + 1j * rng.standard_normal((nt, n))
        h = 1e-6

        def L(a, b):
            return float(dense_loss(torch.tensor(a), torch.tensor(b), it, wt))
        fd = (L(D + h * VD, H + h * VH) - L(D - h * VD, H - h * VH)) / (2 * h)
        an = np.sum(np.real(np.conj(gD) * VD)) + np.sum(np.real(np.conj(gH) * VH))
        assert abs(fd - an) <= 1e-6 * max(1.0, abs(an)), (fd, an)
