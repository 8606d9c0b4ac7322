"""Host-side logic of the nitorch-compatible surface (CPU only): enums,
name normalisation, argument checks and error wording, broadcasting."""
import pytest
import torch

import nitorch_b200 as nb
from nitorch_b200 import api, grid as G, spatial
from nitorch_b200.enums import BoundType, InterpolationType


def test_enum_members_like_reference():
    # nitorch/_C/spatial.cpp:48-73
    assert set(BoundType.__members__) == {
        "replicate", "nearest", "dct1", "mirror", "dct2", "reflect", "dst1", "antimirror",
        "dst2", "antireflect", "dft", "wrap", "zero"}
    assert len(set(BoundType.__members__.values())) == 7
    assert len(set(InterpolationType.__members__.values())) == 8
    assert BoundType.reflect is BoundType.dct2
    assert int(BoundType.zero) == 7 and BoundType.zero.value == 7
    assert BoundType.zero != 7          # pybind11 enums do not compare to ints
    assert int(InterpolationType.cubic) == 3


@pytest.mark.parametrize("name,code", [
    ("replicate", 0), ("border", 0), ("nearest", 0), ("repeat", 0), ("dct1", 1), ("mirror", 1),
    ("dct2", 2), ("reflect", 2), ("reflection", 2), ("neumann", 2), ("dst1", 3), ("antimirror", 3),
    ("dst2", 4), ("antireflect", 4), ("dirichlet", 4), ("dft", 5), ("wrap", 5), ("circular", 5),
    ("zero", 7), ("zeros", 7), ("constant", 7), ("DCT2", 2)])
def test_bound_names(name, code):
    assert int(G.bound_to_nitorch(name, as_type="enum")) == code
    assert G.bound_to_nitorch([name], as_type="enum") == [BoundType(code)]


def test_bound_int_codes_for_prefilter():
    # grid.py:133 maps to the prefilter's codes (_ts/bounds.py:7-14)
    assert G.bound_to_nitorch(["zero", "replicate", "dct1", "dct2", "dst1", "dst2", "dft"],
                              as_type="int") == [0, 1, 2, 3, 4, 5, 6]
    with pytest.raises(ValueError):
        G.bound_to_nitorch("sliding")


def test_order_names():
    assert G.inter_to_nitorch(["nearest", "linear", 2, "cubic", InterpolationType.fourth, 5, "sixth",
                               "seventh"], as_type="int") == list(range(8))
    assert G.inter_to_nitorch(3, as_type="str") == "cubic"
    with pytest.raises(ValueError):
        G.inter_to_nitorch(8)


def test_checks_and_messages():
    x = torch.zeros(1, 1, 4, 4, 4)
    g = torch.zeros(1, 4, 4, 4, 3, dtype=torch.float64)
    with pytest.raises(RuntimeError, match=r"\(\): expected input_opt and grid_opt to have the same dtype"):
        spatial.grid_pull(x, g, [BoundType.dct2], [InterpolationType.linear], 0)
    g = torch.zeros(1, 4, 4, 4, 2)
    with pytest.raises(RuntimeError, match="in last dimension"):
        spatial.grid_pull(x, g, [BoundType.dct2], [InterpolationType.linear], 0)
    g = torch.zeros(1, 4, 4, 4, 3)
    with pytest.raises(RuntimeError, match="non empty parameter bound_mode"):
        spatial.grid_pull(x, g, [], [InterpolationType.linear], 0)
    with pytest.raises(RuntimeError, match="no CPU backend"):
        spatial.grid_pull(x, g, [BoundType.dct2], [InterpolationType.linear], 0)
    with pytest.raises(RuntimeError, match="same batch, width, height"):
        spatial.grid_push(torch.zeros(1, 1, 3, 4, 4), g, [], [BoundType.dct2],
                          [InterpolationType.linear], 0)
    # 16-bit images may pair with float32 grids (stored 16-bit, computed fp32)
    with pytest.raises(RuntimeError, match="no CPU backend"):
        spatial.grid_pull(x.bfloat16(), g, [BoundType.dct2], [InterpolationType.linear], 0)


def test_fold_broadcasting():
    grid = torch.zeros(2, 1, 5, 6, 3)
    inp = torch.zeros(3, 7, 8, 9)          # channel 3, no leading dimension
    g, i, lay = api._fold(grid, inp)
    assert g.shape == (2, 5, 6, 1, 3) or g.shape == (2, 1, 5, 6, 3)
    assert i.shape == (2, 3, 7, 8, 9)
    assert lay.chan == (3,) and lay.lead == (2,)
    assert api._Layout((2,), (3,), 3).restore(torch.zeros(2, 3, 1, 5, 6)).shape == (2, 3, 1, 5, 6)
    grid = torch.zeros(5, 6, 7, 3)
    inp = torch.zeros(5, 6, 7)             # no channel, no leading dimension
    g, i, lay = api._fold(grid, inp)
    assert g.shape == (1, 5, 6, 7, 3) and i.shape == (1, 1, 5, 6, 7)
    assert lay.restore(torch.zeros(1, 1, 5, 6, 7)).shape == (5, 6, 7)
    # leading dimensions broadcast; an image without channel gets a singleton one back
    g, i, lay = api._fold(torch.zeros(4, 1, 2, 3, 2), torch.zeros(5, 2, 3))
    assert g.shape == (4, 2, 3, 2) and i.shape == (4, 5, 2, 3) and lay.chan == (5,)
    g, i, lay = api._fold(torch.zeros(4, 2, 3, 2), torch.zeros(2, 3))
    assert i.shape == (4, 1, 2, 3) and lay.chan == (1,) and lay.lead == (4,)
    assert lay.restore(torch.zeros(4, 1, 2, 3)).shape == (4, 1, 2, 3)
    # push broadcasts the spatial shapes too
    g, i, lay = api._fold(torch.zeros(1, 4, 2), torch.zeros(2, 3, 1), shared_space=True)
    assert g.shape == (1, 3, 4, 2) and i.shape == (1, 2, 3, 4)
    # count: grid only
    g, _, lay = api._fold(torch.zeros(2, 3, 4, 5, 3))
    assert g.shape == (2, 3, 4, 5, 3) and lay.chan == (1,)
    assert lay.restore(torch.zeros(2, 1, 3, 4, 5)).shape == (2, 1, 3, 4, 5)


def test_identity_grid():
    g = nb.identity_grid((3, 4), dtype=torch.float64)
    assert g.shape == (3, 4, 2)
    assert g[2, 3].tolist() == [2.0, 3.0]


def test_install_registers_backend_module():
    import sys
    saved = {k: sys.modules.get(k) for k in ("nitorch._C.spatial", "interpol", "interpol.coeff")}
    try:
        mod = nb.install(set_env=False)
        assert sys.modules["nitorch._C.spatial"] is mod is spatial
        from interpol.coeff import spline_coeff_nd  # noqa: F401
        from interpol.bounds import BoundType as TSB
        assert TSB.dct2.value == 3
    finally:
        for k, v in saved.items():
            if v is None:
                sys.modules.pop(k, None)
            else:
                sys.modules[k] = v


def test_patch_callers_dispatches_by_device():
    """patch_callers replaces nitorch.spatial's callers by dispatchers: CUDA
    tensors go to this package, other tensors to the original function."""
    import types

    import torch

    from nitorch_b200 import integration
    calls = []
    fake = types.ModuleType("fake_spatial")
    for name in ("exp", "resize", "reslice", "grid_jacobian", "grid_jacdet"):
        setattr(fake, name, (lambda n: (lambda x, *a, **k: calls.append(n) or n))(name))
    patched = integration.patch_callers(fake)
    assert sorted(patched) == sorted(["exp", "resize", "reslice", "grid_jacobian", "grid_jacdet"])
    assert fake.exp(torch.zeros(2, 2, 1)) == "exp" and calls == ["exp"]
    assert fake.grid_jacdet(torch.zeros(1, 2, 2, 2)) == "grid_jacdet"
    assert integration.patch_callers(fake) == []  # idempotent


def test_torch_library_ops_fake_shapes():
    """The custom operators are registered and propagate shapes on fake
    tensors (what torch.compile traces with), no GPU needed."""
    import torch
    from torch._subclasses.fake_tensor import FakeTensorMode

    import nitorch_b200.ops  # noqa: F401  (registers the operators)
    with FakeTensorMode():
        x = torch.empty(2, 3, 8, 9, 10)
        g = torch.empty(2, 5, 6, 7, 3)
        y = torch.ops.nitorch_b200.grid_pull(x, g, [2], [3], 0)
        assert y.shape == (2, 3, 5, 6, 7)
        assert torch.ops.nitorch_b200.grid_push(y, g, [8, 9, 10], [2], [3], 0).shape == x.shape
        assert torch.ops.nitorch_b200.grid_push(y, g, [], [2], [3], 0).shape == y.shape
        assert torch.ops.nitorch_b200.grid_count(g, [], [2], [1], 0).shape == (2, 1, 5, 6, 7)
        assert torch.ops.nitorch_b200.grid_grad(x, g, [2], [1], 0).shape == (2, 3, 5, 6, 7, 3)
        gi, gg = torch.ops.nitorch_b200.grid_pull_backward(y, x, g, [2], [3], 0, True, True)
        assert gi.shape == x.shape and gg.shape == g.shape
        assert torch.ops.nitorch_b200.spline_coeff_nd(x, [3], [3], 3).shape == x.shape
