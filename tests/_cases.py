"""Shared seeded test-case generators (CPU, numpy / torch)."""
import numpy as np

BOUNDS = {"replicate": 0, "dct1": 1, "dct2": 2, "dst1": 3, "dst2": 4, "dft": 5, "zero": 7}
BOUND_CODES = list(BOUNDS.values())
ORDERS = list(range(8))


def rng(seed):
    return np.random.default_rng(seed)


def identity(shape):
    mesh = np.meshgrid(*[np.arange(s, dtype=np.float64) for s in shape], indexing="ij")
    return np.stack(mesh, -1)


def make_case(dim, seed, in_size=5, out_size=4, C=2, N=1, spread=1.5):
    """Volume (N,C,*in) ~ N(0,1) and grid (N,*out,dim) = scaled identity +
    N(0, spread) displacement (so samples cover borders and the outside)."""
    r = rng(seed)
    ishape = (in_size,) * dim
    oshape = (out_size,) * dim
    vol = r.standard_normal((N, C) + ishape)
    base = identity(oshape) * ((in_size - 1) / max(out_size - 1, 1))
    grid = base[None] + spread * r.standard_normal((N,) + oshape + (dim,))
    grid = np.repeat(grid, 1, 0)
    return vol, grid


def config1_inputs(size=64):
    """Config-1 workload (seeded, float64 numpy): x, grid, y."""
    from nitorch_b200 import workloads
    x, grid, y = workloads.config1(size)
    return x.numpy(), grid.numpy(), y.numpy()


def sort_keys(grid, src):
    """Source-voxel key of every sampling point of `grid` ((N, *spatial, D)
    numpy), as the source-sorted order defines it: batch item, then the
    linear index of floor(coords) clamped into the source (last axis fastest)."""
    D = grid.shape[-1]
    N = grid.shape[0]
    src = np.array(src)
    c = np.floor(grid.reshape(N, -1, D).astype(np.float64))
    c = np.where(np.isnan(c), 0, c)
    c = np.clip(c, 0, src - 1).astype(np.int64)
    lin = np.zeros(c.shape[:2], np.int64)
    for d in range(D):
        lin = lin * src[d] + c[..., d]
    n = np.arange(N)[:, None]
    return (n * np.prod(src) + lin).reshape(-1)
