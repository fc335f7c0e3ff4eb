"""Stencil feature operators on the B200 (the operators of SurfaceStencilDevice).

Composition follows ``src/cat_surface_gpu/surface_stencil.py:282-644``;
every numeric step is a native kernel from ``csrc/features.cu``.  The only
host synchronisation is the one the reference also makes: reading the mean
edge length to derive the heat-kernel iteration count (``_heat_parameters``).
"""

from __future__ import annotations

from collections import OrderedDict
import math

import numpy as np
import torch

from . import _native
from .surface_stencil import SurfaceStencil, SurfaceStencilDevice

# Device topology tables of the meshes used most recently, as least-recently-used caches: a
# stream of many subjects keeps the shared resampling sphere's tables and the last 32 meshes'
# (a batch of 16 subjects and its template fit) instead of every mesh it has seen.
_CACHE_ENTRIES = 32
_TOPOLOGY_CACHE: OrderedDict = OrderedDict()
_TOPOLOGY_BY_ID: OrderedDict = OrderedDict()
_FACES_BY_ID: OrderedDict = OrderedDict()


def _cache_get(cache: OrderedDict, key):
    hit = cache.get(key)
    if hit is not None:
        cache.move_to_end(key)
    return hit


def _cache_put(cache: OrderedDict, key, value) -> None:
    cache[key] = value
    cache.move_to_end(key)
    while len(cache) > _CACHE_ENTRIES:
        cache.popitem(last=False)


def _shared_faces(faces) -> bool:
    """A read-only int32 face array (the shared resampling sphere): caches may key on its identity."""

    return isinstance(faces, np.ndarray) and not faces.flags.writeable and faces.dtype == np.int32 \
        and faces.flags.c_contiguous


def _stable_order(keys: np.ndarray, n_keys: int) -> np.ndarray:
    """``np.argsort(keys, kind="stable")`` for keys in [0, n_keys): with 16-bit keys numpy's
    stable sort is a radix sort, several times faster on meshes of up to 65,536 vertices."""

    if n_keys <= 1 << 16:
        return np.argsort(keys.astype(np.uint16), kind="stable")
    return np.argsort(keys, kind="stable")


def _topology(faces: np.ndarray, n_points: int, device: torch.device):
    ident = (id(faces), n_points, device.type, device.index) if _shared_faces(faces) else None
    if ident is not None:
        hit = _cache_get(_TOPOLOGY_BY_ID, ident)
        if hit is not None and hit[0] is faces:
            return hit[1]
    f = np.ascontiguousarray(faces, dtype=np.int32)
    key = (device.type, device.index, f.shape, n_points, f.tobytes())
    cached = _cache_get(_TOPOLOGY_CACHE, key)
    if cached is not None:
        if ident is not None:
            _cache_put(_TOPOLOGY_BY_ID, ident, (faces, cached))
        return cached
    lib = _native.library()
    off = np.zeros(n_points + 1, dtype=np.int32)
    nbr = np.zeros(max(1, 6 * f.shape[0]), dtype=np.int32)
    count = _native.check(lib.csg_mesh_neighbours(n_points, f.ctypes.data, f.shape[0], off.ctypes.data,
                                                  nbr.ctypes.data, nbr.size), "csg_mesh_neighbours")
    nbr = nbr[: max(1, count)]
    # per-vertex incidences sorted by (corner, face): the reference's three index_add_ passes.
    # The entries are laid out corner-major with faces ascending, so a stable sort by vertex keeps that order.
    vertex = f.T.reshape(-1)
    corner = np.repeat(np.arange(3, dtype=np.int32), f.shape[0])
    face = np.tile(np.arange(f.shape[0], dtype=np.int32), 3)
    order = _stable_order(vertex, n_points)
    inc = ((face[order] << 2) | corner[order]).astype(np.int32)
    inc_off = np.concatenate(([0], np.cumsum(np.bincount(vertex, minlength=n_points)))).astype(np.int32)
    tensors = tuple(torch.from_numpy(a).to(device) for a in (off, nbr, inc_off, inc))
    max_degree = int(np.diff(off).max()) if n_points else 0
    cached = tensors + (max_degree,)
    _cache_put(_TOPOLOGY_CACHE, key, cached)
    if ident is not None:
        _cache_put(_TOPOLOGY_BY_ID, ident, (faces, cached))
    return cached


def _device_faces(faces, device: torch.device) -> torch.Tensor:
    """Faces on the device; one shared read-only copy for the shared resampling faces."""

    if _shared_faces(faces):
        ident = (id(faces), device.type, device.index)
        hit = _cache_get(_FACES_BY_ID, ident)
        if hit is not None and hit[0] is faces:
            return hit[1]
        tensor = torch.from_numpy(faces.copy()).to(device)
        _cache_put(_FACES_BY_ID, ident, (faces, tensor))
        return tensor
    return torch.as_tensor(np.ascontiguousarray(faces, dtype=np.int32), device=device).contiguous()


def upload_stencil(stencil: SurfaceStencil, device: torch.device, geometry_dtype: torch.dtype,
                   weight_dtype: torch.dtype) -> SurfaceStencilDevice:
    if weight_dtype != torch.float64:
        raise ValueError("stencil weights are float64")
    off, nbr, inc_off, inc, max_degree = _topology(stencil.faces, stencil.sphere_points.shape[0], device)

    pinned = getattr(stencil, "pinned", None)

    def up(array, dtype):
        # copy as stored and convert on the device (the same IEEE rounding as on the host)
        array = np.asarray(array)
        if pinned is not None and array.flags.c_contiguous:
            offset = array.ctypes.data - pinned.data_ptr()
            if 0 <= offset and offset + array.nbytes <= pinned.numel():
                # a view of the page-locked block: an asynchronous copy that torch's pinned-memory
                # cache tracks (the block is not reused before the copy has run)
                source = pinned[offset: offset + array.nbytes].view(torch.from_numpy(array[:0]).dtype)
                return source.reshape(array.shape).to(device, non_blocking=True).to(dtype).contiguous()
        host = torch.from_numpy(np.ascontiguousarray(array, dtype=array.dtype.newbyteorder("=")))
        return host.to(device).to(dtype).contiguous()

    st = SurfaceStencilDevice(
        sphere_points=up(stencil.sphere_points, geometry_dtype),
        faces=_device_faces(stencil.faces, device),
        surface_indices=up(stencil.surface_indices, torch.int32),
        surface_weights=up(stencil.surface_weights, torch.float64),
        sheet_indices=up(stencil.sheet_indices, torch.int32),
        sheet_weights=up(stencil.sheet_weights, torch.float64),
        nx=int(stencil.nx),
        ny=int(stencil.ny),
        source_points=int(stencil.source_points),
        unit_sphere_points=None
        if stencil.unit_sphere_points is None
        else up(stencil.unit_sphere_points, torch.float32),
        neighbour_offsets=off,
        neighbour_indices=nbr,
        max_degree=max_degree,
    )
    st._cache["incidence"] = (inc_off, inc)
    return st


def _stream(operand: torch.Tensor) -> int:
    """The current stream, after checking that ``operand`` lives on the current device."""

    return _native.stream_handle(like=operand)


def _scratch(st: SurfaceStencilDevice, series: int = 1) -> torch.Tensor:
    key = ("scratch", series)
    buf = st._cache.get(key)
    if buf is None:
        n = int(st.sphere_points.shape[0])
        need = _native.library().csg_feature_scratch_bytes(n, int(st.faces.shape[0]), int(st.neighbour_indices.numel()),
                                                          series)
        buf = torch.empty(int(need), dtype=torch.uint8, device=st.sphere_points.device)
        st._cache[key] = buf
    return buf


def resample_vertices(st: SurfaceStencilDevice, vertices) -> torch.Tensor:
    value = torch.as_tensor(vertices, device=st.sphere_points.device)
    if value.ndim != 2 or tuple(value.shape) != (st.source_points, 3):
        raise ValueError(f"vertices shape must be {(st.source_points, 3)}, got {tuple(value.shape)}")
    if value.dtype not in (torch.float32, torch.float64):
        value = value.to(torch.float64)
    value = value.contiguous()
    out = torch.empty((st.surface_indices.shape[0], 3), dtype=value.dtype, device=value.device)
    dtype = _native.CSG_DTYPE_F32 if value.dtype == torch.float32 else _native.CSG_DTYPE_F64
    _native.check(_native.library().csg_feature_resample(dtype, int(out.shape[0]), st.surface_indices.data_ptr(),
                                                         st.surface_weights.data_ptr(), value.data_ptr(),
                                                         out.data_ptr(), _stream(out)), "csg_feature_resample")
    return out


def map_values_to_sheet(st: SurfaceStencilDevice, values) -> torch.Tensor:
    value = torch.as_tensor(values, device=st.sphere_points.device).reshape(-1).to(torch.float64).contiguous()
    if value.numel() != st.sphere_points.shape[0]:
        raise ValueError(f"values must contain {st.sphere_points.shape[0]} elements, got {value.numel()}")
    out = torch.empty((st.ny, st.nx), dtype=torch.float64, device=value.device)
    _native.check(_native.library().csg_feature_sheet_map(st.nx * st.ny, st.sheet_indices.data_ptr(),
                                                          st.sheet_weights.data_ptr(), value.data_ptr(),
                                                          out.data_ptr(), _stream(out)), "csg_feature_sheet_map")
    return out


def _edge_mean(st: SurfaceStencilDevice, vertices: torch.Tensor) -> float:
    """Mean edge length of the stencil's faces on these vertices (reference 347-356); synchronises."""

    v = vertices.contiguous()
    dtype = _native.CSG_DTYPE_F32 if v.dtype == torch.float32 else _native.CSG_DTYPE_F64
    scratch = _scratch(st)
    total = st._cache.setdefault("edge_sum", torch.empty(1, dtype=torch.float64, device=v.device))
    _native.check(_native.library().csg_feature_edge_sum(dtype, int(st.faces.shape[0]), st.faces.data_ptr(), v.data_ptr(),
                                                         total.data_ptr(), scratch.data_ptr(), scratch.numel(),
                                                         _stream(scratch)), "csg_feature_edge_sum")
    return float(total.item()) / (3.0 * int(st.faces.shape[0]))


def edge_means(pairs) -> list[float]:
    """Mean edge lengths of several (stencil, vertices) pairs with one synchronisation.

    Equal to ``_edge_mean`` of each pair: the edge sums widen every coordinate
    to float64, so a float32 geometry and its float64 copy give the same value.
    """

    totals = []
    for st, vertices in pairs:
        v = vertices.contiguous()
        dtype = _native.CSG_DTYPE_F32 if v.dtype == torch.float32 else _native.CSG_DTYPE_F64
        scratch = _scratch(st)
        total = torch.empty(1, dtype=torch.float64, device=v.device)
        _native.check(_native.library().csg_feature_edge_sum(dtype, int(st.faces.shape[0]), st.faces.data_ptr(),
                                                             v.data_ptr(), total.data_ptr(), scratch.data_ptr(),
                                                             scratch.numel(), _stream(scratch)), "csg_feature_edge_sum")
        totals.append(total)
    if not totals:
        return []
    values = torch.cat(totals).cpu().tolist()
    return [float(t) / (3.0 * int(st.faces.shape[0])) for t, (st, _) in zip(values, pairs)]


def _heat_from_edge_mean(edge_mean: float, fwhm: float) -> tuple[int, float]:
    if not (math.isfinite(edge_mean) and edge_mean > 0.0):
        raise ValueError(f"heat kernel: the mean edge length is {edge_mean} (a collapsed or non-finite surface)")
    raw = float(fwhm) * float(fwhm) * 0.541011 / (edge_mean * edge_mean)
    iterations = max(1, int(math.ceil(raw)))
    sigma = float(fwhm) * 0.7355345 / float(iterations ** 0.5)
    return iterations, sigma


def heat_parameters(st: SurfaceStencilDevice, vertices: torch.Tensor, fwhm: float) -> tuple[int, float]:
    """Iteration count and sigma of the iterative heat kernel (reference 359-369)."""

    return _heat_from_edge_mean(_edge_mean(st, vertices), fwhm)


def smooth_geometry(st: SurfaceStencilDevice, vertices, fwhm: float, edge_mean: float | None = None) -> torch.Tensor:
    value = torch.as_tensor(vertices, device=st.sphere_points.device).to(torch.float32).contiguous()
    if edge_mean is None:
        edge_mean = _edge_mean(st, value)
    iterations, _ = _heat_from_edge_mean(edge_mean, fwhm)
    out = torch.empty_like(value)
    scratch = _scratch(st)
    _native.check(_native.library().csg_feature_smooth_geometry(
        int(value.shape[0]), st.neighbour_offsets.data_ptr(), st.neighbour_indices.data_ptr(), value.data_ptr(),
        iterations, out.data_ptr(), scratch.data_ptr(), scratch.numel(), _stream(scratch)), "csg_feature_smooth_geometry")
    return out


def _smooth_series(st, values, geometry, fwhms, via_norm: bool, edge_mean: float | None = None) -> torch.Tensor:
    n = int(st.sphere_points.shape[0])
    base = torch.as_tensor(values, device=st.sphere_points.device).to(torch.float64).reshape(-1).contiguous()
    if base.numel() != n:
        raise ValueError("values must have shape [sphere_points]")
    geom = torch.as_tensor(geometry, device=st.sphere_points.device).contiguous()
    if tuple(geom.shape) != (n, 3):
        raise ValueError("vertices must have shape [sphere_points, 3]")
    if geom.dtype not in (torch.float32, torch.float64):
        geom = geom.to(torch.float64)
    if edge_mean is None:  # one reduction and one synchronisation for every FWHM of the series
        edge_mean = _edge_mean(st, geom)
    params = [_heat_from_edge_mean(edge_mean, f) for f in fwhms]
    counts = ctypes_int_array([p[0] for p in params])
    sigmas = _native.doubles([p[1] for p in params])
    out = torch.empty((len(fwhms), n), dtype=torch.float64, device=base.device)
    scratch = _scratch(st, len(fwhms))
    dtype = _native.CSG_DTYPE_F32 if geom.dtype == torch.float32 else _native.CSG_DTYPE_F64
    import ctypes

    _native.check(_native.library().csg_feature_smooth_values(
        n, st.neighbour_offsets.data_ptr(), st.neighbour_indices.data_ptr(), int(st.neighbour_indices.numel()), dtype,
        geom.data_ptr(), base.data_ptr(), len(fwhms), ctypes.addressof(sigmas), ctypes.addressof(counts),
        int(via_norm), out.data_ptr(), scratch.data_ptr(), scratch.numel(), _stream(scratch)), "csg_feature_smooth_values")
    return out


def ctypes_int_array(values):
    import ctypes

    values = [int(v) for v in values]
    return (ctypes.c_int32 * len(values))(*values)


def smooth_values(st, values, vertices, fwhm: float) -> torch.Tensor:
    """One FWHM (reference 390-412): distances through a vector norm, then squared."""

    return _smooth_series(st, values, vertices, (float(fwhm),), True)[0]


def smooth_values_many(st, values, vertices, fwhms) -> tuple[torch.Tensor, ...]:
    """Several FWHMs in one batched smoothing (reference 414-476): squared distances summed."""

    if not fwhms:
        return ()
    geometry = torch.as_tensor(vertices, device=st.sphere_points.device).to(torch.float64)
    out = _smooth_series(st, values, geometry, tuple(fwhms), False)
    return tuple(out[i] for i in range(len(fwhms)))


def vertex_normals(st: SurfaceStencilDevice, vertices) -> torch.Tensor:
    geometry = torch.as_tensor(vertices, device=st.sphere_points.device).to(torch.float32).contiguous()
    inc_off, inc = st._cache["incidence"]
    out = torch.empty_like(geometry)
    _native.check(_native.library().csg_feature_vertex_normals(int(geometry.shape[0]), st.faces.data_ptr(),
                                                               inc_off.data_ptr(), inc.data_ptr(), geometry.data_ptr(),
                                                               out.data_ptr(), _stream(out)), "csg_feature_vertex_normals")
    return out


def _minmax(st: SurfaceStencilDevice, values: torch.Tensor) -> torch.Tensor:
    v = values.contiguous()
    rows = 1 if v.ndim == 1 else int(v.shape[0])
    n = v.numel() // rows
    out = torch.empty_like(v)
    scratch = _scratch(st, max(1, rows))
    _native.check(_native.library().csg_feature_minmax(n, rows, v.data_ptr(), out.data_ptr(), scratch.data_ptr(),
                                                       scratch.numel(), _stream(scratch)), "csg_feature_minmax")
    return out


def _type5_base(st: SurfaceStencilDevice, geometry: torch.Tensor, edge_mean: float | None = None) -> torch.Tensor:
    smoothed = smooth_geometry(st, geometry, 50.0, edge_mean)
    normals = vertex_normals(st, smoothed)
    out = torch.empty(int(geometry.shape[0]), dtype=torch.float64, device=geometry.device)
    _native.check(_native.library().csg_feature_normal_displacement(int(geometry.shape[0]), smoothed.data_ptr(),
                                                                    geometry.data_ptr(), normals.data_ptr(),
                                                                    out.data_ptr(), _stream(out)),
                  "csg_feature_normal_displacement")
    return out


def curvature_type5(st: SurfaceStencilDevice, vertices, fwhm: float) -> torch.Tensor:
    geometry = torch.as_tensor(vertices, device=st.sphere_points.device).to(torch.float32).contiguous()
    values = _smooth_series(st, _type5_base(st, geometry), geometry, (float(fwhm),), True)[0]
    return _minmax(st, values)


def curvature_type5_to_sheet_many(st: SurfaceStencilDevice, vertices, fwhms,
                                  edge_mean: float | None = None) -> tuple[torch.Tensor, ...]:
    """Type-5 curvature sheets for several FWHMs; ``edge_mean`` (of ``vertices``, from
    :func:`edge_means`) saves the synchronisation that computes it."""

    if not fwhms:
        return ()
    geometry = torch.as_tensor(vertices, device=st.sphere_points.device).to(torch.float32).contiguous()
    if edge_mean is None:
        edge_mean = _edge_mean(st, geometry)
    base = _type5_base(st, geometry, edge_mean)
    # the same geometry in float64: the same edge mean
    smoothed = _smooth_series(st, base, geometry.to(torch.float64), tuple(fwhms), False, edge_mean)
    normalised = _minmax(st, smoothed)
    maps = torch.stack([map_values_to_sheet(st, normalised[i]).reshape(-1) for i in range(len(fwhms))])
    maps = _minmax(st, maps)
    return tuple(maps[i].reshape(st.ny, st.nx) for i in range(len(fwhms)))


def curvature_type2(st: SurfaceStencilDevice, vertices, fwhm: float) -> torch.Tensor:
    geometry = torch.as_tensor(vertices, device=st.sphere_points.device).to(torch.float32).contiguous()
    normals = vertex_normals(st, geometry)
    values = torch.empty(int(geometry.shape[0]), dtype=torch.float64, device=geometry.device)
    _native.check(_native.library().csg_feature_curvature2(int(geometry.shape[0]), st.neighbour_offsets.data_ptr(),
                                                           st.neighbour_indices.data_ptr(), geometry.data_ptr(),
                                                           normals.data_ptr(), values.data_ptr(), _stream(values)),
                  "csg_feature_curvature2")
    values = _smooth_series(st, values, geometry, (float(fwhm),), True)[0]
    return _minmax(st, values)


def curvature_to_sheet(st: SurfaceStencilDevice, vertices, fwhm: float, curvtype: int = 5) -> torch.Tensor:
    if curvtype == 5:
        values = curvature_type5(st, vertices, fwhm)
    elif curvtype == 2:
        values = curvature_type2(st, vertices, fwhm)
    else:
        raise NotImplementedError("The GPU surface backend supports only upstream curvtype 2 and 5")
    return _minmax(st, map_values_to_sheet(st, values).reshape(-1)).reshape(st.ny, st.nx)
