"""Seeded synthetic workloads of the push/pull benchmark configurations.

The reference publishes no dataset for this path; these generators stand in
with the shapes, sizes and value distributions of the benchmark
configurations.  Inputs are drawn on the CPU in float64 from
``torch.Generator().manual_seed(seed)``; Gaussian smoothing is a separable
float64 convolution with dct2 (mirror-about-edge) padding, truncated at 4
sigma; displacement fields are rescaled after smoothing to the stated
standard deviation.  Callers cast / move the results.

  config1 : 1x1x64^3 U[0,1) volume, identity + smoothed N(0,2) displacement
            (sigma 4, std 2), order 1, dct2, extrapolate=False.
  config2 : 1x3x192^3 smoothed N(0,1) (sigma 2), identity + smoothed
            displacement (std ~4, ~5 % of samples outside), order 3, dct2,
            prefilter.
  config3 : 4x8x512^2 (2-D) / 2x1x128^3 (3-D) U[0,1) with random affine
            grids (rotation <= 15 deg, scale 0.9-1.1, shift <= 10 vox),
            shift rescaled to put ~10 % of samples outside.
  config4 : 64 volumes, each axis U{96..256}, C U{1..4}, orders 1 / 3
            alternating, dct2, identity + smoothed displacement (sigma 4,
            std 2).
  config5 : stationary velocity 1x160x192x160x3 smoothed N(0,1) (sigma 3)
            and moving / fixed images 1x1x160x192x160.
"""
import math

import torch


def _gen(seed):
    return torch.Generator().manual_seed(int(seed))


def gaussian_kernel(sigma):
    r = int(math.ceil(4 * sigma))
    x = torch.arange(-r, r + 1, dtype=torch.float64)
    k = torch.exp(-0.5 * (x / sigma) ** 2)
    return k / k.sum()


def smooth(x, sigma, ndim):
    """Separable Gaussian smoothing of the last `ndim` dims (dct2 padding)."""
    if sigma <= 0:
        return x
    k = gaussian_kernel(sigma).to(x)
    r = (k.numel() - 1) // 2
    shape = x.shape
    for d in range(ndim):
        ax = x.dim() - ndim + d
        y = x.movedim(ax, -1)
        s = y.shape
        y = y.reshape(-1, 1, s[-1])
        n = s[-1]
        # mirror about the edge, repeated if the radius exceeds the length
        idx = torch.arange(-r, n + r)
        p = 2 * n
        idx = idx % p
        idx = torch.where(idx >= n, p - 1 - idx, idx)
        y = y[..., idx]
        y = torch.nn.functional.conv1d(y, k.view(1, 1, -1))
        x = y.reshape(s).movedim(-1, ax)
    assert x.shape == shape
    return x


def identity_grid(shape, dtype=torch.float64):
    mesh = torch.meshgrid(*[torch.arange(s, dtype=dtype) for s in shape], indexing="ij")
    return torch.stack(mesh, -1)


def smooth_displacement(shape, sigma, std, seed, batch=1):
    dim = len(shape)
    g = _gen(seed)
    d = torch.randn((batch, dim, *shape), generator=g, dtype=torch.float64)
    d = smooth(d, sigma, dim)
    d = d * (std / d.std())
    return d.movedim(1, -1).contiguous()


def oob_fraction(grid, shape, tol=0.05):
    inb = torch.ones(grid.shape[:-1], dtype=torch.bool)
    for a, n in enumerate(shape):
        c = grid[..., a]
        inb &= (c >= -tol) & (c < n - 1 + tol)
    return 1.0 - inb.double().mean().item()


def config1(size=64):
    shape = (size,) * 3
    x = torch.rand((1, 1, *shape), generator=_gen(1), dtype=torch.float64)
    grid = identity_grid(shape)[None] + smooth_displacement(shape, 4.0, 2.0, seed=2)
    y = torch.rand((1, 1, *shape), generator=_gen(3), dtype=torch.float64)
    return x, grid, y


def config2(size=192, channels=3, disp_std=4.0):
    shape = (size,) * 3
    x = torch.randn((1, channels, *shape), generator=_gen(11), dtype=torch.float64)
    x = smooth(x, 2.0, 3)
    x = x / x.std()
    grid = identity_grid(shape)[None] + smooth_displacement(shape, 2.0, disp_std, seed=12)
    return x, grid


def affine_grid_2d3d(shape, batch, seed, oob_target=0.10):
    """Random affine grids about the FOV centre; the shift is rescaled
    (bisection) until ~`oob_target` of the samples fall outside."""
    dim = len(shape)
    g = _gen(seed)
    c = torch.tensor([(s - 1) / 2 for s in shape], dtype=torch.float64)
    base = identity_grid(shape)
    grids = []
    for _ in range(batch):
        ang = (torch.rand(3 if dim == 3 else 1, generator=g, dtype=torch.float64) * 2 - 1) * math.radians(15)
        scl = 0.9 + 0.2 * torch.rand(dim, generator=g, dtype=torch.float64)
        sh = (torch.rand(dim, generator=g, dtype=torch.float64) * 2 - 1) * 10
        if dim == 2:
            ca, sa = math.cos(ang[0]), math.sin(ang[0])
            Rm = torch.tensor([[ca, -sa], [sa, ca]], dtype=torch.float64)
        else:
            Rm = torch.eye(3, dtype=torch.float64)
            for ax, a in enumerate(ang.tolist()):
                ca, sa = math.cos(a), math.sin(a)
                i, j = [k for k in range(3) if k != ax]
                Q = torch.eye(3, dtype=torch.float64)
                Q[i, i], Q[i, j], Q[j, i], Q[j, j] = ca, -sa, sa, ca
                Rm = Rm @ Q
        A = Rm * scl
        lin = (base - c) @ A.T + c

        def frac(t):
            return oob_fraction(lin + t * sh, shape)
        lo, hi = 0.0, 1.0
        while frac(hi) < oob_target and hi < 64:
            hi *= 2
        for _ in range(30):
            mid = 0.5 * (lo + hi)
            if frac(mid) < oob_target:
                lo = mid
            else:
                hi = mid
        grids.append(lin + hi * sh)
    return torch.stack(grids)


def config3(dim):
    if dim == 2:
        shape, N, C = (512, 512), 4, 8
    else:
        shape, N, C = (128, 128, 128), 2, 1
    x = torch.rand((N, C, *shape), generator=_gen(21), dtype=torch.float64)
    grid = affine_grid_2d3d(shape, N, seed=22)
    return x, grid


def config4(n_volumes=64, lo=96, hi=256, seed=31):
    """List of (x (1,C,*shape), grid (1,*shape,3), order) items."""
    g = _gen(seed)
    items = []
    for v in range(n_volumes):
        shape = tuple(int(s) for s in torch.randint(lo, hi + 1, (3,), generator=g))
        C = int(torch.randint(1, 5, (1,), generator=g))
        order = 1 if v % 2 == 0 else 3
        items.append((shape, C, order, int(torch.randint(0, 2**31 - 1, (1,), generator=g))))
    return items


def config4_volume(shape, C, vseed):
    """Materialise one config-4 volume (float64, CPU)."""
    x = torch.rand((1, C, *shape), generator=_gen(vseed), dtype=torch.float64)
    # smoothing a 256^3 displacement in float64 is slow on CPU; a coarse
    # field upsampled by linear interpolation has the same character
    coarse = tuple(max(4, s // 4) for s in shape)
    d = torch.randn((1, 3, *coarse), generator=_gen(vseed + 1), dtype=torch.float64)
    d = smooth(d, 1.0, 3)
    d = torch.nn.functional.interpolate(d, size=shape, mode="trilinear", align_corners=True)
    d = d * (2.0 / d.std())
    grid = identity_grid(shape)[None] + d.movedim(1, -1)
    return x, grid.contiguous()


def config5(shape=(160, 192, 160)):
    v = torch.randn((1, *shape, 3), generator=_gen(41), dtype=torch.float64)
    v = smooth(v.movedim(-1, 1), 3.0, 3).movedim(1, -1).contiguous()
    mov = smooth(torch.randn((1, 1, *shape), generator=_gen(42), dtype=torch.float64), 3.0, 3)
    fix = smooth(torch.randn((1, 1, *shape), generator=_gen(43), dtype=torch.float64), 3.0, 3)
    return v, mov, fix
