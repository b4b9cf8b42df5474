"""
Seeded synthetic catalogues: lognormal data and uniform randoms in a box.

These stand in for the mock catalogues the reference's tests build with
mockfactory (pyrecon/tests/utils.py:25-80), which are not available here.
The recipe, with k in h/Mpc:

* a Gaussian field G on an n^3 grid covering the box, with power spectrum
  P(k) ~ k^-1.5 exp(-(8 k)^2), made by colouring white noise in Fourier space
  and rescaled so that std(G) = sigma_G;
* a lognormal density 1 + delta = exp(G - sigma_G^2 / 2);
* exactly ``size`` data points whose cells are drawn independently with
  probability proportional to 1 + delta (a multinomial draw, done by
  inverting the cumulative sum), uniform within their cell;
* randoms uniform in the box; weights 1 or uniform in [wmin, wmax].

``backend='numpy'`` draws with ``numpy.random.default_rng(seed)``;
``backend='torch'`` draws on a torch device with a seeded ``torch.Generator``
(fast at nmesh 512 and tens of millions of points).  The two back-ends give
catalogues with the same statistics, not the same numbers.
"""

import numpy as np


def _power(k):
    with np.errstate(divide='ignore'):
        pk = np.where(k > 0, k ** -1.5 * np.exp(-(8. * k) ** 2), 0.)
    return pk


def gaussian_field_numpy(nmesh, boxsize, sigma=0.8, seed=1000):
    rng = np.random.default_rng(seed)
    white = rng.standard_normal((nmesh,) * 3)
    wk = np.fft.rfftn(white)
    kf = 2 * np.pi / boxsize
    kx = np.fft.fftfreq(nmesh, d=1. / nmesh) * kf
    kz = np.fft.rfftfreq(nmesh, d=1. / nmesh) * kf
    k = np.sqrt(kx[:, None, None] ** 2 + kx[None, :, None] ** 2 + kz[None, None, :] ** 2)
    wk *= np.sqrt(_power(k))
    field = np.fft.irfftn(wk, s=(nmesh,) * 3)
    field *= sigma / field.std()
    return field


def lognormal_positions_numpy(size, nmesh, boxsize, boxcenter, sigma=0.8, seed=2000, field_seed=1000, dtype='f8'):
    field = gaussian_field_numpy(nmesh, boxsize, sigma=sigma, seed=field_seed)
    density = np.exp(field - sigma ** 2 / 2.).ravel()
    cdf = np.cumsum(density)
    rng = np.random.default_rng(seed)
    cells = np.searchsorted(cdf, rng.uniform(0., cdf[-1], size), side='right')
    cells = np.minimum(cells, nmesh ** 3 - 1)
    ijk = np.stack(np.unravel_index(cells, (nmesh,) * 3), axis=-1).astype('f8')
    cell = boxsize / nmesh
    offset = np.asarray(boxcenter, dtype='f8') - boxsize / 2.
    positions = offset + (ijk + rng.uniform(0., 1., (size, 3))) * cell
    return positions.astype(dtype)


def uniform_positions_numpy(size, boxsize, boxcenter, seed=3000, dtype='f8'):
    rng = np.random.default_rng(seed)
    offset = np.asarray(boxcenter, dtype='f8') - boxsize / 2.
    return (offset + rng.uniform(0., boxsize, (size, 3))).astype(dtype)


def weights_numpy(size, low=0.5, high=1.5, seed=4000, dtype='f8'):
    if low == high:
        return np.full(size, low, dtype=dtype)
    return np.random.default_rng(seed).uniform(low, high, size).astype(dtype)


# ---------------------------------------------------------------------------------------------
# torch back-end (device-side generation for large catalogues)
# ---------------------------------------------------------------------------------------------

def _torch_generator(seed, device):
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    return g


def gaussian_field_torch(nmesh, boxsize, sigma=0.8, seed=1000, device='cuda'):
    import torch
    g = _torch_generator(seed, device)
    white = torch.randn((nmesh,) * 3, generator=g, device=device, dtype=torch.float32)
    wk = torch.fft.rfftn(white)
    del white
    kf = 2 * np.pi / boxsize
    kx = torch.fft.fftfreq(nmesh, d=1. / nmesh, device=device) * kf
    kz = torch.fft.rfftfreq(nmesh, d=1. / nmesh, device=device) * kf
    k = torch.sqrt(kx[:, None, None] ** 2 + kx[None, :, None] ** 2 + kz[None, None, :] ** 2)
    amp = torch.where(k > 0, k.clamp_min(1e-30) ** -0.75 * torch.exp(-0.5 * (8. * k) ** 2), torch.zeros_like(k))
    wk *= amp
    del k, amp
    field = torch.fft.irfftn(wk, s=(nmesh,) * 3)
    del wk
    field *= sigma / field.std()
    return field


def lognormal_positions_torch(size, nmesh, boxsize, boxcenter, sigma=0.8, seed=2000, field_seed=1000,
                              dtype='f8', device='cuda'):
    import torch
    field = gaussian_field_torch(nmesh, boxsize, sigma=sigma, seed=field_seed, device=device)
    density = torch.exp(field.double() - sigma ** 2 / 2.).reshape(-1)
    del field
    cdf = torch.cumsum(density, 0)
    del density
    g = _torch_generator(seed, device)
    u = torch.rand(size, generator=g, device=device, dtype=torch.float64) * cdf[-1]
    cells = torch.searchsorted(cdf, u, right=True).clamp_max(nmesh ** 3 - 1)
    del cdf, u
    iz = cells % nmesh
    iy = (cells // nmesh) % nmesh
    ix = cells // (nmesh * nmesh)
    ijk = torch.stack([ix, iy, iz], dim=-1).double()
    cell = boxsize / nmesh
    offset = torch.as_tensor(np.asarray(boxcenter, dtype='f8') - boxsize / 2., device=device)
    jitter = torch.rand((size, 3), generator=g, device=device, dtype=torch.float64)
    positions = offset + (ijk + jitter) * cell
    return positions.to(getattr(torch, np.dtype(dtype).name))


def uniform_positions_torch(size, boxsize, boxcenter, seed=3000, dtype='f8', device='cuda'):
    import torch
    g = _torch_generator(seed, device)
    offset = torch.as_tensor(np.asarray(boxcenter, dtype='f8') - boxsize / 2., device=device)
    positions = offset + torch.rand((size, 3), generator=g, device=device, dtype=torch.float64) * boxsize
    return positions.to(getattr(torch, np.dtype(dtype).name))


def weights_torch(size, low=0.5, high=1.5, seed=4000, dtype='f8', device='cuda'):
    import torch
    tdtype = getattr(torch, np.dtype(dtype).name)
    if low == high:
        return torch.full((size,), low, dtype=tdtype, device=device)
    g = _torch_generator(seed, device)
    return (low + (high - low) * torch.rand(size, generator=g, device=device, dtype=torch.float64)).to(tdtype)
