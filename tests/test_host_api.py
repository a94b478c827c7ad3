"""Host-side mirror of Partia's API: catalog naming and slots, input
promotion and validation, LinRange axes, frames, sample geometry."""
import math

import numpy as np
import pytest

import partia_b200 as P
from partia_b200 import workloads as W


def test_catalog_names_slots_and_shepard_flags():
    # InterpolationCatalog.jl:141-230
    cat = P.InterpolationCatalog.from_columns(("rho", "T", "vx", "vy", "vz"), scalars=("rho", "T"), gradients=("T",),
                                              divergences=("v",), curls=("v",))
    assert cat.ordered_names == ("rho", "T", "∇Tˣ", "∇Tʸ", "∇Tᶻ", "∇⋅v", "∇×vˣ", "∇×vʸ", "∇×vᶻ")
    assert cat.scalar_slots == (1, 2) and cat.grad_slots == (2,)
    assert cat.div_slots == ((3, 4, 5),) and cat.curl_slots == ((3, 4, 5),)
    assert cat.scalar_snormalization == (False, True)
    c = cat.concise()
    assert list(c.scalars) == [0, 1] and list(c.grads) == [1] and list(c.divs) == [2, 3, 4]
    assert c.L == 9
    cat2 = P.InterpolationCatalog.from_columns(("ρ",), scalars=("ρ",))
    assert cat2.scalar_snormalization == (False,)


def test_catalog_errors():
    with pytest.raises(P.ArgumentError):
        P.InterpolationCatalog.from_columns(("a", "a"), scalars=("a",))
    with pytest.raises(KeyError):
        P.InterpolationCatalog.from_columns(("a",), scalars=("b",))
    with pytest.raises(P.DimensionMismatch):
        P.InterpolationCatalog(scalar_names=("a",), scalar_slots=())


def test_input_validation_and_promotion():
    n = 5
    x = np.zeros(n, dtype=np.float32)
    with pytest.raises(P.DimensionMismatch):
        P.InterpolationInput(x, x, x[:3], x, x, x)
    inp, cat = P.build_input(P.B200ComputeBackend(), x, x, x, np.zeros(n), x, x, (np.zeros(n, np.float32),),
                             column_names=("a",), scalars=("a",))
    assert inp.dtype == np.float64 and inp.quant[0].dtype == np.float64
    inp32, _ = P.build_input(P.B200ComputeBackend(), x, x, x, x, x, x, (x,), column_names=("a",))
    assert inp32.dtype == np.float32


def test_linrange_is_julia_lerp():
    # collect(LinRange(a, b, n))[i] = (1 - t) a + t b, t = (i-1)/(n-1)
    a, b, n = 1 / 128, 127 / 128, 64
    ax = P.linrange(a, b, n)
    t = np.arange(n) / (n - 1)
    assert np.array_equal(ax, (1 - t) * a + t * b)
    assert ax[0] == a and ax[-1] == b
    g = P.StructuredGrid.cartesian((0.2, 0.7, 3), (0.25, 0.55, 2), (0.3, 0.6, 2))
    c = g.coordinate_grid()
    assert len(c[0]) == 12 and c[0][1] == g.axes[0][1] and c[1][3] == g.axes[1][1]  # x fastest


def test_flatten_restore_roundtrip():
    g = P.StructuredGrid.cartesian((0.0, 1.0, 4), (0.0, 2.0, 3), (0.0, 3.0, 2))
    flat = P.flatten(P.Cartesian, g)
    flat.grid[:] = np.arange(len(flat.grid))
    back = P.restore_struct(P.Cartesian, flat, g.axes)
    assert back.grid.shape == (4, 3, 2) and back.grid[1, 0, 0] == 1 and back.grid[0, 1, 0] == 4
    with pytest.raises(P.ArgumentError):
        P.restore_struct(P.Cartesian, flat, (g.axes[0] + 1, g.axes[1], g.axes[2]))


def test_frame_rotation_conventions():
    # Frame(x, f0, u0): r0 = f0 x u0; rotate!(yaw, pitch, roll) right-multiplies
    # rotations about the initial u0, r0, f0 (Frames/operations/rotation.jl:15-26)
    fr = W.Frame((0.0, 0.0, 0.0), (0.0, 0.0, -1.0), (0.0, 1.0, 0.0))
    assert np.allclose(fr.right(), [1.0, 0.0, 0.0])
    fr.rotate(math.pi / 2, 0.0, 0.0)  # yaw 90 deg about +y
    assert np.allclose(fr.forward(), [-1.0, 0.0, 0.0], atol=1e-15)
    assert np.allclose(fr.up(), [0.0, 1.0, 0.0], atol=1e-15)
    fr2 = W.c3_frame()
    B = np.stack([fr2.right(), fr2.up(), fr2.forward()])
    assert np.allclose(B @ B.T, np.eye(3), atol=1e-14)  # orthonormal
    with pytest.raises(ValueError):
        W.Frame((0, 0, 0), (1, 0, 0), (1, 1, 0))


def test_plane_and_box_coordinates_layout():
    fr = W.Frame((0.5, 0.5, 0.5), (0.0, 0.0, 1.0), (0.0, 1.0, 0.0)).as_array()
    x, y, z = W.plane_coordinates(fr, (-0.5, 0.5, 3), (-1.0, 1.0, 2))
    # k = i + (j-1) nx: first row varies along frame right
    assert len(x) == 6 and np.allclose(z, 0.5)
    bx = W.box_coordinates(fr, (-0.5, 0.5, 3), (-1.0, 1.0, 2), (0.0, 0.2, 2))
    assert len(bx[0]) == 12


def test_workload_generators_are_seeded():
    a = W.plummer_c2(n=1000, seed=1)
    b = W.plummer_c2(n=1000, seed=1)
    assert np.array_equal(a["x"], b["x"]) and np.all(np.sqrt(a["x"] ** 2 + a["y"] ** 2 + a["z"] ** 2) <= 1.0)
    c = W.clumps(2000, seed=2)
    assert len(c["x"]) == 2000 and c["m"].sum() == pytest.approx(1.0)


def test_hs_follows_the_call_pointers_on_the_host():
    """Context._hs: for a call with host pointers, hs becomes a contiguous
    host array of the context dtype (lists, scalars and tensors alike)."""
    import types

    import torch
    from partia_b200.engine import Context
    fake = types.SimpleNamespace(dtype=np.dtype(np.float64), device=0)
    assert Context._hs(fake, 1, None, False) is None
    a = Context._hs(fake, 1, [0.1, 0.2], False)
    assert isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags.c_contiguous
    assert np.array_equal(a, [0.1, 0.2])
    assert np.array_equal(Context._hs(fake, 2, 0.05, False), [0.05])
    t = torch.tensor([0.25, 0.5], dtype=torch.float32)
    b = Context._hs(fake, 1, t, False)
    assert isinstance(b, np.ndarray) and b.dtype == np.float64 and np.array_equal(b, [0.25, 0.5])
    fake32 = types.SimpleNamespace(dtype=np.dtype(np.float32), device=0)
    assert Context._hs(fake32, 1, np.array([0.1, 0.2]), False).dtype == np.float32
