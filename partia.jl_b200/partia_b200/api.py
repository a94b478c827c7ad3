"""Partia's interpolation API over the B200 library.

Names, argument meaning and error behaviour follow Partia.jl so that code
written against Partia's CPU/CUDA backends reads the same here:

  build_input                      interpolation_setup/constructor.jl:68-136
  InterpolationInput               interpolation_setup/InterpolationInput.jl:41-107
  InterpolationCatalog             interpolation_setup/InterpolationCatalog.jl:9-230
  itpGather/itpScatter/itpSymmetric interpolation_setup/InterpolationStrategy.jl:3-5
  LinearBVH_ (LinearBVH!)          interpolation_setup/InterpolationInput.jl:201-221
  matches_lbvh_leaf_order          interpolation_setup/InterpolationInput.jl:265-267
  initialize_interpolation         grid_interpolation/setup/initialize_interpolation.jl:39-55,100-111
  PointSamples_interpolation       grid_interpolation/drivers/PointSamples_driver.jl:34-48,98-118
  LineSamples_interpolation        grid_interpolation/drivers/LineSamples_driver.jl:39-55,116-141
  StructuredGrid_interpolation     grid_interpolation/drivers/StructuredGrid_driver.jl:46-64
  PointSamples / LineSamples / StructuredGrid / GridBundle   src/julia/Grids/

(paths relative to src/julia/KernelInterpolation/ unless stated).  The
compute path is libpartia_b200 only; there is no CPU fallback.
"""
from __future__ import annotations

import numpy as np

from . import _lib as L
from .engine import CatalogC, Context


# ---------------------------------------------------------------------------
# errors (Julia exception names)
# ---------------------------------------------------------------------------
class ArgumentError(ValueError):
    pass


class DimensionMismatch(ValueError):
    pass


# ---------------------------------------------------------------------------
# backends, strategies, kernels
# ---------------------------------------------------------------------------
class AbstractExecutionBackend:
    pass


class B200ComputeBackend(AbstractExecutionBackend):
    """Backend singleton of the B200 path (device index, precision mode)."""

    def __init__(self, device: int = 0, precision: int = L.PSB_PREC_FP64):
        self.device = device
        self.precision = precision


class AbstractInterpolationStrategy:
    code = -1


class itpGather(AbstractInterpolationStrategy):
    code = L.PSB_GATHER


class itpScatter(AbstractInterpolationStrategy):
    code = L.PSB_SCATTER


class itpSymmetric(AbstractInterpolationStrategy):
    code = L.PSB_SYMMETRIC


class AbstractSPHKernel:
    """Kernel families of kernel_function/kernels/*.jl; code = psb_kernel."""
    code = None


class M4_spline(AbstractSPHKernel):
    code = L.PSB_KERNEL_M4


class M5_spline(AbstractSPHKernel):
    code = L.PSB_KERNEL_M5


class M6_spline(AbstractSPHKernel):
    code = L.PSB_KERNEL_M6


class C2_Wendland(AbstractSPHKernel):
    code = L.PSB_KERNEL_C2


class C4_Wendland(AbstractSPHKernel):
    code = L.PSB_KERNEL_C4


class C6_Wendland(AbstractSPHKernel):
    code = L.PSB_KERNEL_C6


# ---------------------------------------------------------------------------
# InterpolationInput / InterpolationCatalog / build_input
# ---------------------------------------------------------------------------
class InterpolationInput:
    """Particle columns of one float type (InterpolationInput.jl:41-107)."""

    def __init__(self, x, y, z, m, h, rho, quant=(), smoothed_kernel=M5_spline):
        arrs = [np.asarray(a) for a in (x, y, z, m, h, rho)]
        Np = len(arrs[3])
        for d, a in enumerate(arrs[:3]):
            if len(a) != Np:
                raise DimensionMismatch(f"coord[{d + 1}] length {len(a)} != Nparticles {Np}")
        if len(arrs[4]) != Np:
            raise DimensionMismatch(f"h length {len(arrs[4])} != Nparticles {Np}")
        if len(arrs[5]) != Np:
            raise DimensionMismatch(f"ρ length {len(arrs[5])} != Nparticles {Np}")
        quant = tuple(np.asarray(q) for q in quant)
        for j, q in enumerate(quant):
            if len(q) != Np:
                raise DimensionMismatch(f"quant[{j + 1}] length {len(q)} != Nparticles {Np}")
        self.Npart = Np
        self.smoothed_kernel = smoothed_kernel
        self.coord = tuple(arrs[:3])
        self.m, self.h, self.rho = arrs[3], arrs[4], arrs[5]
        self.quant = quant
        # the device context that holds this input's particles and LBVH, and
        # the LBVH last built from it (kept across driver calls)
        self._b200_ctx = None
        self._b200_lbvh = None

    def __deepcopy__(self, memo):
        """A copy of the arrays; the copy gets its own device state when used."""
        import copy
        return InterpolationInput(*[copy.deepcopy(a, memo) for a in (*self.coord, self.m, self.h, self.rho)],
                                  tuple(copy.deepcopy(q, memo) for q in self.quant),
                                  smoothed_kernel=self.smoothed_kernel)

    @property
    def dtype(self):
        return self.m.dtype

    def __len__(self):
        return self.Npart


_DERIV = ("ˣ", "ʸ", "ᶻ")


class InterpolationCatalog:
    """Requested outputs resolved to column slots (InterpolationCatalog.jl:9-230).

    Slots are 1-based as in the reference; a grad slot of 0 requests the
    gradient of the particle density itself.
    """

    def __init__(self, scalar_names=(), scalar_slots=(), grad_names=(), grad_slots=(), div_names=(), div_slots=(),
                 curl_names=(), curl_slots=()):
        if len(scalar_slots) != len(scalar_names):
            raise DimensionMismatch(f"scalar_slots length {len(scalar_slots)} != scalar_names length {len(scalar_names)}")
        if len(grad_slots) != len(grad_names):
            raise DimensionMismatch(f"grad_slots length {len(grad_slots)} != grad_names length {len(grad_names)}")
        if len(div_slots) != len(div_names):
            raise DimensionMismatch(f"div_slots length {len(div_slots)} != div_names length {len(div_names)}")
        if len(curl_slots) != len(curl_names):
            raise DimensionMismatch(f"curl_slots length {len(curl_slots)} != curl_names length {len(curl_names)}")
        self.scalar_names = tuple(scalar_names)
        self.scalar_slots = tuple(int(s) for s in scalar_slots)
        # Shepard normalisation off only for :ρ / :rho (InterpolationCatalog.jl:222-225)
        self.scalar_snormalization = tuple(n not in ("ρ", "rho") for n in self.scalar_names)
        self.grad_names = tuple(grad_names)
        self.grad_slots = tuple(int(s) for s in grad_slots)
        self.div_names = tuple(div_names)
        self.div_slots = tuple(tuple(int(v) for v in s) for s in div_slots)
        self.curl_names = tuple(curl_names)
        self.curl_slots = tuple(tuple(int(v) for v in s) for s in curl_slots)
        names = list(self.scalar_names)
        for b in self.grad_names:
            names += [f"∇{b}{s}" for s in _DERIV]
        names += [f"∇⋅{b}" for b in self.div_names]
        for b in self.curl_names:
            names += [f"∇×{b}{s}" for s in _DERIV]
        self.ordered_names = tuple(names)

    @classmethod
    def from_columns(cls, column_names, scalars=(), gradients=(), divergences=(), curls=()):
        column_names = tuple(column_names)
        if len(set(column_names)) != len(column_names):
            raise ArgumentError("column_names must be unique")
        idx = {n: i + 1 for i, n in enumerate(column_names)}
        vec = lambda b: tuple(idx[f"{b}{s}"] for s in ("x", "y", "z"))
        return cls(scalar_names=scalars, scalar_slots=tuple(idx[s] for s in scalars),
                   grad_names=gradients, grad_slots=tuple(idx[g] for g in gradients),
                   div_names=divergences, div_slots=tuple(vec(d) for d in divergences),
                   curl_names=curls, curl_slots=tuple(vec(c) for c in curls))

    @property
    def L(self):
        return len(self.ordered_names)

    def concise(self) -> CatalogC:
        """to_concise_catalog, with the library's 0-based slots."""
        return CatalogC(scalars=[s - 1 for s in self.scalar_slots],
                        shepard=[1 if f else 0 for f in self.scalar_snormalization],
                        grads=[s - 1 for s in self.grad_slots],
                        divs=[v - 1 for s in self.div_slots for v in s],
                        curls=[v - 1 for s in self.curl_slots for v in s])


def build_input(backend, x_col, y_col, z_col, m_col, h_col, rho_col, quantity_columns=(), *, column_names=(),
                scalars=(), gradients=(), divergences=(), curls=(), smoothed_kernel=M5_spline):
    """constructor.jl:68-136: promote every column to one float type."""
    cols = [np.asarray(c) for c in (x_col, y_col, z_col, m_col, h_col, rho_col)]
    qc = [np.asarray(c) for c in quantity_columns]
    if len(column_names) != len(qc):
        raise DimensionMismatch("column_names must match quantity_columns one-to-one")
    T = np.result_type(*cols, *qc)
    if not np.issubdtype(T, np.floating):
        T = np.float64
    cv = lambda a: np.array(a, dtype=T, copy=True)
    inp = InterpolationInput(*[cv(c) for c in cols], tuple(cv(q) for q in qc), smoothed_kernel=smoothed_kernel)
    cat = InterpolationCatalog.from_columns(column_names, scalars=scalars, gradients=gradients,
                                            divergences=divergences, curls=curls)
    return inp, cat


# ---------------------------------------------------------------------------
# sample containers
# ---------------------------------------------------------------------------
def _vectors(t):
    """The caller's tuple itself when it already holds arrays, so that
    containers made by similar() share one coordinate tuple, as Julia's do."""
    if isinstance(t, tuple) and all(isinstance(c, np.ndarray) for c in t):
        return t
    return tuple(np.asarray(c) for c in t)


class PointSamples:
    def __init__(self, grid, coor):
        grid = np.asarray(grid)
        for d, c in enumerate(coor):
            if len(c) != len(grid):
                raise DimensionMismatch(f"coor[{d + 1}] length {len(c)} != grid length {len(grid)}")
        self.grid = grid
        self.coor = _vectors(coor)

    def __len__(self):
        return len(self.grid)

    def similar(self):
        return PointSamples(np.zeros_like(self.grid), self.coor)


class LineSamples:
    def __init__(self, grid, origin, direction):
        grid = np.asarray(grid)
        for d in range(3):
            if len(origin[d]) != len(grid) or len(direction[d]) != len(grid):
                raise DimensionMismatch("origin/direction lengths must match the grid length")
        self.grid = grid
        self.origin = _vectors(origin)
        self.direction = _vectors(direction)

    def __len__(self):
        return len(self.grid)

    def similar(self):
        return LineSamples(np.zeros_like(self.grid), self.origin, self.direction)


def linrange(a, b, n, dtype=np.float64):
    """collect(LinRange{T}(a, b, n)): element i is T((1 - t)*a + t*b), t = (i-1)/(n-1)."""
    if n == 1:
        return np.array([a], dtype=dtype)
    j = np.arange(n, dtype=np.float64)
    t = j / float(n - 1)
    a64, b64 = np.float64(dtype(a)), np.float64(dtype(b))
    return ((1.0 - t) * a64 + t * b64).astype(dtype)


class Cartesian:
    pass


class StructuredGrid:
    def __init__(self, grid, axes, size):
        self.grid = grid
        self.axes = tuple(axes)
        self.size = tuple(size)

    @classmethod
    def cartesian(cls, *params, dtype=np.float64):
        """StructuredGrid(Cartesian, (min, max, n)...) (StructuredGrid.jl:234-262)."""
        axes = tuple(linrange(p[0], p[1], p[2], dtype) for p in params)
        size = tuple(int(p[2]) for p in params)
        return cls(np.zeros(size, dtype=dtype, order="F"), axes, size)

    def coordinate_grid(self):
        """Column-major (x fastest) coordinates (StructuredGrid.jl:140-155)."""
        mesh = np.meshgrid(*self.axes, indexing="ij")
        return tuple(m.ravel(order="F") for m in mesh)


class GridBundle:
    def __init__(self, grids, names):
        self.grids = tuple(grids)
        self.names = tuple(names)

    def __getitem__(self, name):
        return self.grids[self.names.index(name)]


def flatten(coord, grid: StructuredGrid) -> PointSamples:
    if coord is not Cartesian:
        raise ArgumentError("only Cartesian structured grids are provided by the B200 backend")
    return PointSamples(np.asarray(grid.grid).ravel(order="F"), grid.coordinate_grid())


def restore_struct(coord, grid: PointSamples, axes, atol=1e-8, rtol=1e-8) -> StructuredGrid:
    size = tuple(len(a) for a in axes)
    expected = StructuredGrid(None, axes, size).coordinate_grid()
    for a, e in zip(grid.coor, expected):
        if not np.allclose(a, e, atol=atol, rtol=rtol):
            raise ArgumentError("PointSamples coordinates do not match the provided axes under Cartesian dispatch")
    return StructuredGrid(np.asarray(grid.grid).reshape(size, order="F"), axes, size)


# ---------------------------------------------------------------------------
# LBVH handle and the drivers
# ---------------------------------------------------------------------------
class LinearBVH:
    """Device-resident LBVH of one InterpolationInput.

    ``leaf_coor`` and ``leaf_scale`` are copies of the Morton-ordered
    coordinates and smoothing lengths, as LinearBVH keeps them
    (LinearBoundingVolumeHierarchy/LinearBVH/LinearBVH.jl:8-14); the tree
    itself lives on the device context ``ctx``.  ``generation`` names the
    build of ``ctx`` this handle describes: a context rebuilt from other
    particles no longer holds this tree.
    """

    def __init__(self, ctx: Context, leaf_coor, leaf_scale, perm, generation: int):
        self.ctx = ctx
        self.leaf_coor = leaf_coor
        self.leaf_scale = leaf_scale
        self.perm = perm
        self.generation = generation

    @property
    def nleaf(self):
        return len(self.leaf_scale)


def _check_kernel(input: InterpolationInput):
    if getattr(input.smoothed_kernel, "code", None) is None:
        raise ArgumentError(f"{input.smoothed_kernel!r} is not a kernel family of this backend")


def _input_context(input: InterpolationInput, backend: B200ComputeBackend) -> Context:
    """The context that holds this input on the backend's device (made once)."""
    ctx = input._b200_ctx
    if ctx is None or ctx.device != backend.device or ctx.h is None:
        ctx = Context(backend.device)
        input._b200_ctx = ctx
    return ctx


def _upload(ctx: Context, input: InterpolationInput):
    ctx.set_particles(*input.coord, input.m, input.h, input.rho, input.quant, kernel=input.smoothed_kernel.code)


def LinearBVH_(input: InterpolationInput, backend: B200ComputeBackend | None = None) -> LinearBVH:
    """LinearBVH!(input): build on the device and permute input in place.

    The build runs on the input's own context, made on first use and kept:
    later builds of the same input reuse its device buffers (no allocation)."""
    backend = backend or B200ComputeBackend()
    _check_kernel(input)
    if input.Npart < 1:
        raise ArgumentError("BinaryRadixTree: enc.codes must be non-empty (got n=0).")
    ctx = _input_context(input, backend)
    _upload(ctx, input)
    perm, _ = ctx.build()
    for a in (*input.coord, input.m, input.h, input.rho, *input.quant):
        a[:] = a[perm]
    ctx.generation += 1
    lbvh = LinearBVH(ctx, tuple(c.copy() for c in input.coord), input.h.copy(), perm, ctx.generation)
    input._b200_lbvh = lbvh
    return lbvh


def matches_lbvh_leaf_order(input: InterpolationInput, lbvh: LinearBVH) -> bool:
    return all(np.array_equal(input.coord[d], lbvh.leaf_coor[d]) for d in range(3)) and np.array_equal(
        input.h, lbvh.leaf_scale)


def _bind(lbvh: LinearBVH, input: InterpolationInput):
    """Put ``input``'s values on ``lbvh``'s context, whose leaf order it matches.

    The tree depends on coordinates and h only, which the leaf-order check
    has compared, so only m, rho and the columns are replaced
    (psb_set_values).  A context rebuilt from other particles since
    ``lbvh`` was made, or set with another kernel or float type, is rebuilt
    from ``input``: its coordinates are already in Morton order, so the build
    permutes nothing."""
    ctx = lbvh.ctx
    _check_kernel(input)
    same = (ctx.generation == lbvh.generation and ctx.kernel == input.smoothed_kernel.code
            and ctx.dtype == np.dtype(input.dtype) and ctx.n == input.Npart)
    if same:
        ctx.set_values(input.m, input.rho, input.quant)
        return
    _upload(ctx, input)
    perm, _ = ctx.build()
    if not np.array_equal(perm, np.arange(input.Npart)):
        raise ArgumentError("Provided LBVH leaf order does not match the current input ordering. "
                            "Ensure the LBVH was built from the same Morton-reordered input.")
    ctx.generation += 1
    lbvh.generation = ctx.generation


def _input_lbvh(backend: B200ComputeBackend, input: InterpolationInput) -> LinearBVH:
    """LinearBVH!(input) as the drivers call it (initialize_interpolation.jl:50).

    An input already in the leaf order of the LBVH last built from it would be
    permuted by the identity and get the same tree again; that LBVH is reused
    with the input's current values instead of being rebuilt."""
    lbvh = input._b200_lbvh
    if (lbvh is not None and lbvh.ctx is input._b200_ctx and lbvh.ctx.h is not None
            and lbvh.ctx.device == backend.device and matches_lbvh_leaf_order(input, lbvh)):
        _bind(lbvh, input)
        return lbvh
    return LinearBVH_(input, backend)


def initialize_interpolation(backend, grid_template, input=None, catalog=None):
    """Allocate outputs, build (or reuse) the LBVH when input is given, concise catalog."""
    if catalog is None:
        input, catalog = None, input
    grids = tuple(grid_template.similar() for _ in range(catalog.L))
    conc = catalog.concise()
    if input is None:
        return grids, catalog.ordered_names, conc
    lbvh = _input_lbvh(backend, input)
    return grids, lbvh, catalog.ordered_names, conc


def _strategy(s):
    if isinstance(s, type) and issubclass(s, AbstractInterpolationStrategy):
        return s.code
    raise ArgumentError(f"unknown interpolation strategy {s!r}")


_LEAF_ORDER_MSG = ("Provided LBVH leaf order does not match the current input ordering. "
                   "Ensure the LBVH was built from the same Morton-reordered input.")


def PointSamples_interpolation(backend, grid_template: PointSamples, input: InterpolationInput, *args,
                               precision=None):
    """PointSamples_interpolation(backend, grid, input, [LBVH,] catalog, itp_strategy=itpSymmetric)."""
    if args and isinstance(args[0], LinearBVH):
        lbvh, catalog = args[0], args[1]
        strategy = args[2] if len(args) > 2 else itpSymmetric
        if not matches_lbvh_leaf_order(input, lbvh):
            raise ArgumentError(_LEAF_ORDER_MSG)
        _bind(lbvh, input)
        grids, names, conc = initialize_interpolation(backend, grid_template, catalog)
    else:
        catalog = args[0]
        strategy = args[1] if len(args) > 1 else itpSymmetric
        grids, lbvh, names, conc = initialize_interpolation(backend, grid_template, input, catalog)
    prec = backend.precision if precision is None else precision
    outs = [g.grid for g in grids]
    lbvh.ctx.interp_points(*grid_template.coor, conc, strategy=_strategy(strategy), hmode=L.PSB_H_NEAREST,
                           prec=prec, out=outs)
    return GridBundle(grids, names)


def LineSamples_interpolation(backend, grid_template: LineSamples, input: InterpolationInput, *args, precision=None):
    """LineSamples_interpolation(backend, lines, input, [LBVH,] catalog, itp_strategy=itpScatter)."""
    if args and isinstance(args[0], LinearBVH):
        lbvh, catalog = args[0], args[1]
        strategy = args[2] if len(args) > 2 else itpScatter
    else:
        lbvh, catalog = None, args[0]
        strategy = args[1] if len(args) > 1 else itpScatter
    if strategy is not itpScatter:
        raise ArgumentError("LineSamples_interpolation only supports itpScatter. Line-integrated samples do not have "
                            "a well-defined query smoothing length ha, so itpGather and itpSymmetric are not "
                            "supported.")
    if catalog.grad_names or catalog.div_names or catalog.curl_names:
        raise ArgumentError("LineSamples_interpolation supports scalar quantities only")
    if lbvh is not None:
        if not matches_lbvh_leaf_order(input, lbvh):
            raise ArgumentError(_LEAF_ORDER_MSG)
        _bind(lbvh, input)
        grids, names, conc = initialize_interpolation(backend, grid_template, catalog)
    else:
        grids, lbvh, names, conc = initialize_interpolation(backend, grid_template, input, catalog)
    prec = backend.precision if precision is None else precision
    outs = [g.grid for g in grids]
    lbvh.ctx.interp_lines(grid_template.origin, grid_template.direction, conc, strategy=L.PSB_SCATTER, prec=prec,
                          out=outs)
    return GridBundle(grids, names)


def StructuredGrid_interpolation(backend, coord, grid_template: StructuredGrid, input: InterpolationInput, catalog,
                                 itp_strategy=itpSymmetric, precision=None):
    """StructuredGrid_driver.jl:46-64 for Cartesian grids.

    The reference flattens the grid into PointSamples, interpolates and
    restores the structure.  Here the column-major sample coordinates are
    generated on the device from the axes (psb_interp_grid), which gives the
    flattened samples' results bit for bit, written straight into the
    column-major output grids."""
    if coord is not Cartesian:
        raise ArgumentError("only Cartesian structured grids are provided by the B200 backend")
    T = np.dtype(input.dtype)
    axes = tuple(np.asarray(a, dtype=T) for a in grid_template.axes)
    size = tuple(len(a) for a in axes)
    names = catalog.ordered_names
    conc = catalog.concise()
    lbvh = _input_lbvh(backend, input)
    prec = backend.precision if precision is None else precision
    flat = [np.empty(int(np.prod(size)), dtype=T) for _ in range(catalog.L)]
    lbvh.ctx.interp_grid(*axes, conc, strategy=_strategy(itp_strategy), hmode=L.PSB_H_NEAREST, prec=prec, out=flat)
    grids = tuple(StructuredGrid(f.reshape(size, order="F"), axes, size) for f in flat)
    return GridBundle(grids, names)
