"""B-spline prefilter vectorised over lines with torch CPU operations -- TEST
AND BASELINE INFRASTRUCTURE, never the product.

The same recursions as the C restatement in pushpull_oracle.c (or_coeff_line,
following nitorch/_C/_ts/coeff.py:34-281: poles :34-57, gain :61-65, initial
conditions dct1 :94-134, dct2 :137-170, dft :69-91, final conditions
:173-215, causal / anticausal passes :254-281), written the way the
reference's own CPU prefilter runs: every step of a recursion is one tensor
operation over all lines of the volume at once (the filtered axis moved to
the front), in the tensor's own dtype, on torch's CPU threads.  It stands in
for the reference's prefilter (the third-party `interpol` package, absent on
the benchmark host) in the timed CPU baseline of the full-size workload,
where the line-by-line C restatement would take seconds per call.  Pinned
against the C restatement in tests/test_golden_oracle.py.
"""
import math

import torch


def _poles(order):
    """B-spline prefilter poles (coeff.py:34-57)."""
    if order in (0, 1):
        return []
    if order == 2:
        return [math.sqrt(8.0) - 3.0]
    if order == 3:
        return [math.sqrt(3.0) - 2.0]
    if order == 4:
        return [math.sqrt(664.0 - math.sqrt(438976.0)) + math.sqrt(304.0) - 19.0,
                math.sqrt(664.0 + math.sqrt(438976.0)) - math.sqrt(304.0) - 19.0]
    if order == 5:
        return [math.sqrt(67.5 - math.sqrt(4436.25)) + math.sqrt(26.25) - 6.5,
                math.sqrt(67.5 + math.sqrt(4436.25)) - math.sqrt(26.25) - 6.5]
    if order == 6:
        return [-0.488294589303044755130118038883789062112279161239377608394,
                -0.081679271076237512597937765737059080653379610398148178525368,
                -0.00141415180832581775108724397655859252786416905534669851652709]
    if order == 7:
        return [-0.5352804307964381655424037816816460718339231523426924148812,
                -0.122554615192326690515272264359357343605486549427295558490763,
                -0.0091486948096082769285930216516478534156925639545994482648003]
    raise ValueError(f"order {order}")


def _trunc(z):
    return int(math.ceil(-30.0 / math.log(abs(z))))


def _weighted(c, w):
    """sum_k w[k] * c[k] over the leading axis (w: python floats)."""
    wt = torch.tensor(w, dtype=c.dtype)
    return torch.tensordot(wt, c[:len(w)], dims=1)


def _init(c, z, kind):
    n = c.shape[0]
    if kind == "dct1":
        m = _trunc(z)
        if m < n:
            return _weighted(c, [z ** k for k in range(m)])
        zn = z ** (n - 1)
        w = [1.0] + [z ** k + zn * zn / z ** k for k in range(1, n - 1)] + [zn]
        return _weighted(c, w) / (1.0 - zn * zn)
    if kind == "dct2":
        zn = z ** n
        zlast = zn * (1.0 + 1.0 / (z + zn * zn))
        w = [1.0] + [z ** k + z ** (2 * n - 1 - k) for k in range(1, n - 1)] + [zlast]
        s = _weighted(c, w)
        return s * (z / (1.0 - zn * zn)) + c[0]
    m = min(_trunc(z), n)  # dft
    rev = torch.flip(c[n - m + 1:], (0,)) if m > 1 else c[:0]
    s = c[0] + (_weighted(rev, [z ** j for j in range(1, m)]) if m > 1 else 0.0)
    return s / (1.0 - z ** m)


def _final(c, z, kind):
    n = c.shape[0]
    if kind == "dct1":
        return (z * c[n - 2] + c[n - 1]) * (z / (z * z - 1.0))
    if kind == "dct2":
        return c[n - 1] * (z / (z - 1.0))
    m = min(_trunc(z), n)
    s = z * c[n - 1]
    if m > 1:
        s = s + _weighted(c, [z ** (j + 2) for j in range(m - 1)])
    return s / (z ** m - 1.0)


_KIND = {0: "dct1", 2: "dct1", 1: "dct2", 3: "dct2", 6: "dft"}


def spline_coeff(x, bound_ts, order, dim=-1):
    """Interpolating coefficients along axis `dim` of the CPU tensor `x`
    (new tensor, x's dtype).  bound_ts: the prefilter's integer codes
    (0 zero, 1 replicate, 2 dct1, 3 dct2, 6 dft)."""
    poles = _poles(order)
    if bound_ts not in _KIND:
        raise NotImplementedError("prefilter bound not implemented")
    c = x.movedim(dim, 0).clone()
    n = c.shape[0]
    if not poles or n == 1:
        return c.movedim(0, dim)
    kind = _KIND[bound_ts]
    gain = 1.0
    for z in poles:
        gain *= (1.0 - z) * (1.0 - 1.0 / z)
    c.mul_(gain)
    for z in poles:
        c[0] = _init(c, z, kind)
        for i in range(1, n):
            c[i].add_(c[i - 1], alpha=z)
        c[n - 1] = _final(c, z, kind)
        for i in range(n - 2, -1, -1):
            c[i] = (c[i + 1] - c[i]) * z
    return c.movedim(0, dim).contiguous()


def spline_coeff_nd(x, bound_ts, order, dim):
    """The last `dim` axes, one bound / order per axis (lists padded with
    their last entry)."""
    b = list(bound_ts) + [bound_ts[-1]] * dim
    o = list(order) + [order[-1]] * dim
    for d in range(dim):
        x = spline_coeff(x, b[d], o[d], dim=x.dim() - dim + d)
    return x
