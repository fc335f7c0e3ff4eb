"""CPU tests for the Surf2Sphere path: oracle pinning, topology, schedule, ABI."""

from __future__ import annotations

import math
import re

import numpy as np
import pytest

from conftest import ROOT, load_surf2sphere_golden
from oracle import areal as oracle


def _tetrahedron():
    vertices = np.asarray(((1, 1, 1), (-1, -1, 1), (-1, 1, -1), (1, -1, -1)), dtype=np.float32)
    faces = np.asarray(((0, 1, 2), (0, 3, 1), (0, 2, 3), (1, 3, 2)), dtype=np.int32)
    return vertices, faces


# --- oracle pinned against the upstream binary's own outputs -----------------


@pytest.mark.parametrize("case", ["c1", "c2"])
def test_oracle_matches_upstream_binary(case):
    """prefix (binary stop_at=5) + oracle sweeps + ellipsoid step == binary stop_at=10 within 1e-3."""

    g = load_surf2sphere_golden(case)
    prefix = g["prefix"]
    radius = float(np.sqrt(np.max(np.sum(prefix.astype(np.float64) ** 2, axis=1))))
    smoothed = oracle.areal_sweeps(prefix, g["faces"], iterations=5000, project_every=1000, radius=radius)
    final = oracle.ellipsoid_to_sphere(smoothed, g["source_area"])
    stats = oracle.error_stats(g["final"], final)
    assert stats["max"] <= 1e-3 and stats["p99"] <= 1e-3 and stats["mean"] <= 1e-3, stats
    # The restatement is far tighter than the contract (measured 1.5e-5 / 3.1e-5).
    assert stats["max"] <= 1e-4, stats


def test_oracle_modes_agree_on_tetrahedron():
    v, f = _tetrahedron()
    out_cat = oracle.areal_sweeps(v, f, iterations=10, project_every=3, radius=2.0)
    out_64 = oracle.areal_sweeps(v.astype(np.float64), f, iterations=10, project_every=3, radius=2.0, arithmetic="fp64")
    np.testing.assert_allclose(out_cat, out_64, atol=1e-5)


def test_ellipsoid_projection_radius():
    """Same check as the reference's test_surf2sphere.py:61-77."""

    from cat_surface_gpu_b200.gifti import GiftiMesh
    from cat_surface_gpu_b200.surf2sphere import convert_ellipsoid_to_sphere_with_surface_area, surface_area

    v, f = _tetrahedron()
    area = surface_area(GiftiMesh(v, f))
    projected = convert_ellipsoid_to_sphere_with_surface_area(v, area)
    radius = np.linalg.norm(projected.astype(np.float64), axis=1)
    np.testing.assert_allclose(radius, math.sqrt(area / (4.0 * math.pi)), rtol=0.0, atol=2.0e-6)
    np.testing.assert_array_equal(projected, oracle.ellipsoid_to_sphere(v, area))


# --- host topology builders ---------------------------------------------------


def test_topology_groups_match_oracle_and_are_independent(native_library):
    from cat_surface_gpu_b200 import synthetic
    from cat_surface_gpu_b200.gifti import GiftiMesh
    from cat_surface_gpu_b200.surf2sphere import Surf2SphereTopology

    v, f = synthetic.folded_icosphere(3, seed=4)
    topo = Surf2SphereTopology.from_mesh(GiftiMesh(v, f))
    levels = oracle.dependency_levels(v.shape[0], f)
    assert len(topo.ordered_groups) == levels.max() + 1
    for level, group in enumerate(topo.ordered_groups):
        np.testing.assert_array_equal(group, np.flatnonzero(levels == level))
    edges = set()
    for a, b, c in f.tolist():
        edges |= {(a, b), (b, a), (b, c), (c, b), (a, c), (c, a)}
    for groups in (topo.color_groups, topo.ordered_groups):
        covered = np.sort(np.concatenate(groups))
        np.testing.assert_array_equal(covered, np.arange(v.shape[0]))
        for group in groups:
            members = set(group.tolist())
            assert not any((a in members and b in members) for a, b in edges)
    # incident faces ascending per vertex and complete
    for vertex in range(v.shape[0]):
        row = topo.incident_faces[vertex, topo.incident_mask[vertex]]
        np.testing.assert_array_equal(row, np.flatnonzero((f == vertex).any(axis=1)))


def test_tetrahedron_topology_like_reference(native_library):
    """Reference test_surf2sphere.py:36-58 on the same tetrahedron."""

    from cat_surface_gpu_b200.gifti import GiftiMesh
    from cat_surface_gpu_b200.surf2sphere import Surf2SphereTopology

    v, f = _tetrahedron()
    topo = Surf2SphereTopology.from_mesh(GiftiMesh(v, f))
    assert topo.incident_faces.shape == (4, 3)
    assert topo.incident_mask.all()
    assert len(topo.color_groups) >= 4
    assert len(topo.ordered_groups) >= 1


def test_bad_faces_raise(native_library):
    from cat_surface_gpu_b200.gifti import GiftiMesh
    from cat_surface_gpu_b200.surf2sphere import Surf2SphereTopology

    v, f = _tetrahedron()
    bad = f.copy()
    bad[1, 2] = 7
    with pytest.raises(ValueError):
        Surf2SphereTopology.from_mesh(GiftiMesh(v, bad))


# --- the wavefront schedule is race-free (host simulation of the kernel) -----


def _simulate_wavefront(plan, faces, n, iterations, project_every):
    """Replay the kernel's step arithmetic and check every read's sweep version.

    version[v] is the sweep whose value vertex v currently holds.  At a step,
    vertex v of (epoch-local) sweep s must read: itself at s-1, lower
    neighbours at s, higher neighbours at s-1 -- exactly the sequential
    Gauss-Seidel order -- and no two vertices updated in one step may share a
    face.  Returns the number of updates performed.
    """

    slot_off, slot_tri = plan.slot_off, plan.slot_tri
    version = np.zeros(n, dtype=np.int64)
    L, D = plan.n_levels, plan.level_stride
    level_of = np.full(n, -1, dtype=np.int64)
    for level in range(L):
        level_of[plan.order[plan.level_begin[level] : plan.level_end[level]]] = level
    assert (level_of >= 0).all()
    updates = 0
    last = iterations - 1
    start = 1
    global_sweep = 0
    while start <= last:
        end = last if project_every <= 0 else min(last, ((start - 1) // project_every + 1) * project_every)
        S = end - start + 1
        for t in range(0, (S - 1) * D + L):
            r = t % D
            hi = min(t, L - 1)
            hi -= (hi - r) % D
            lo = max(r, t - (S - 1) * D)
            lo += (r - lo) % D
            if hi < lo:
                continue
            active = plan.order[plan.level_begin[lo] : plan.level_end[hi]]
            snapshot = version.copy()
            for v in active.tolist():
                assert (t - level_of[v]) % D == 0
                sweep = global_sweep + (t - level_of[v]) // D + 1
                assert snapshot[v] == sweep - 1
                for slot in range(slot_off[v], slot_off[v + 1]):
                    for u in slot_tri[slot, :3].tolist():
                        if u == v:
                            continue
                        expected = sweep if u < v else sweep - 1
                        assert snapshot[u] == expected, (v, u, sweep, snapshot[u])
                version[v] = sweep
                updates += 1
            # no face shared by two vertices of the same step
            members = set(active.tolist())
            for v in members:
                for slot in range(slot_off[v], slot_off[v + 1]):
                    assert not (set(slot_tri[slot, :3].tolist()) - {v}) & members
        global_sweep += S
        assert (version == global_sweep).all()
        start = end + 1
    return updates


@pytest.mark.parametrize("subdivisions,iterations,project", [(1, 7, 3), (2, 6, 0), (2, 9, 4)])
def test_wavefront_schedule_reads_sequential_versions(native_library, subdivisions, iterations, project):
    from cat_surface_gpu_b200 import synthetic
    from cat_surface_gpu_b200.surf2sphere import SweepPlan

    v, f = synthetic.folded_icosphere(subdivisions, seed=3)
    # scramble vertex ids so the level structure is less regular
    perm = np.random.default_rng(5).permutation(v.shape[0])
    inverse = np.argsort(perm)
    f = inverse[f].astype(np.int32)
    plan = SweepPlan.build(f, v.shape[0])
    updates = _simulate_wavefront(plan, f, v.shape[0], iterations, project)
    assert updates == v.shape[0] * (iterations - 1)


def test_plan_schedule_is_a_valid_tight_potential(native_library):
    """Plan groups f(v) satisfy 1 <= f(w) - f(v) <= stride - 1 on every edge v < w, with a stride no larger
    than the longest-path levels give (6 instead of 11 on the 61,442-vertex hull)."""

    g = load_surf2sphere_golden("c2")
    from cat_surface_gpu_b200.surf2sphere import SweepPlan

    n = g["prefix"].shape[0]
    f = g["faces"]
    plan = SweepPlan.build(f, n)
    np.testing.assert_array_equal(np.sort(plan.order), np.arange(n))  # every vertex once
    group = np.full(n, -1, dtype=np.int64)
    for level in range(plan.n_levels):
        group[plan.order[plan.level_begin[level] : plan.level_end[level]]] = level
    assert (group >= 0).all()
    edges = np.sort(np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]]), axis=1)
    gap = group[edges[:, 1]] - group[edges[:, 0]]
    assert gap.min() >= 1 and gap.max() <= plan.level_stride - 1
    levels = oracle.dependency_levels(n, f)
    longest_path_stride = int((levels[edges[:, 1]] - levels[edges[:, 0]]).max()) + 1
    assert plan.level_stride <= longest_path_stride
    assert (longest_path_stride, plan.level_stride) == (11, 6)
    # groups of one residue class mod the stride are contiguous in `order`
    residues = [group[plan.order[i]] % plan.level_stride for i in range(n)]
    assert residues == sorted(residues)


# --- the C ABI loads and exports every declared symbol ----------------------


def test_library_exports_every_header_symbol(native_library):
    header = (ROOT / "include" / "catsurf_b200.h").read_text()
    names = re.findall(r"CSG_API\s+[\w\s\*]+?\b(csg_\w+)\s*\(", header)
    assert len(names) >= 10
    for name in names:
        assert hasattr(native_library, name), name
    assert native_library.csg_abi_version() >= 1


def test_gifti_round_trip(tmp_path):
    from cat_surface_gpu_b200.gifti import GiftiMesh, read_gifti_mesh, write_gifti_mesh, write_vertices_like

    v, f = _tetrahedron()
    write_gifti_mesh(tmp_path / "a.gii", GiftiMesh(v, f))
    mesh = read_gifti_mesh(tmp_path / "a.gii")
    np.testing.assert_array_equal(mesh.vertices, v)
    np.testing.assert_array_equal(mesh.faces, f)
    write_vertices_like(tmp_path / "a.gii", tmp_path / "b.gii", v * 2)
    other = read_gifti_mesh(tmp_path / "b.gii")
    np.testing.assert_array_equal(other.faces, f)
    np.testing.assert_array_equal(other.vertices, v * 2)


def test_gifti_large_arrays_parallel_deflate_and_payload_reuse(tmp_path):
    """Large arrays deflate in parallel chunks into one standard zlib stream; a face array
    equal to one decoded before reuses its stored payload; any other array is encoded anew."""

    import base64
    import re
    import zlib

    from conftest import GOLDEN

    from cat_surface_gpu_b200 import gifti
    from cat_surface_gpu_b200.gifti import GiftiMesh, read_gifti_mesh, write_gifti_mesh, write_vertices_like

    c = np.load(GOLDEN / "surf2sphere_c2.npz")
    v, f = c["surface"].astype(np.float32), c["faces"].astype(np.int32)
    for raw in (v.tobytes(), f.tobytes(), v[:5000].tobytes()):
        z, lengths = gifti._deflate(raw, 1)
        assert zlib.decompress(z) == raw
        assert zlib.decompressobj().decompress(z) == raw
        text = base64.b64encode(z)

        def native(index):
            out = np.empty(len(raw), dtype=np.uint8)
            assert gifti._decode_payload(text, True, index, out) == zlib.adler32(raw)
            return out.tobytes()

        # the chunk index inflates the chunks apart to the same bytes; an index that does not
        # fit the stream falls back to one inflate, and a wrong one fails the check
        assert native(lengths) == raw
        assert (lengths is None) == (len(raw) < gifti._PARALLEL_MIN)
        if lengths:
            assert native(lengths[:-1]) == raw
            bad = [lengths[0] + 1, lengths[1] - 1] + lengths[2:]
            with pytest.raises(ValueError):
                native(bad)
    write_gifti_mesh(tmp_path / "a.gii", GiftiMesh(v, f))
    a = read_gifti_mesh(tmp_path / "a.gii")
    np.testing.assert_array_equal(a.vertices, v)
    np.testing.assert_array_equal(a.faces, f)

    def payloads(path):
        return re.findall(r"<Data>([^<]*)</Data>", (tmp_path / path).read_text())

    moved = (v * 1.5).astype(np.float32)
    write_gifti_mesh(tmp_path / "b.gii", GiftiMesh(moved, a.faces.copy()), reference_path=tmp_path / "a.gii")
    assert payloads("b.gii")[1] == payloads("a.gii")[1]  # the decoded face payload, reused
    b = read_gifti_mesh(tmp_path / "b.gii")
    np.testing.assert_array_equal(b.vertices, moved)
    np.testing.assert_array_equal(b.faces, f)
    changed = a.faces.copy()
    changed[7] = changed[7][::-1]
    write_gifti_mesh(tmp_path / "c.gii", GiftiMesh(moved, changed))
    np.testing.assert_array_equal(read_gifti_mesh(tmp_path / "c.gii").faces, changed)
    write_vertices_like(tmp_path / "a.gii", tmp_path / "d.gii", moved)
    assert payloads("d.gii")[1] == payloads("a.gii")[1]  # copied from the reference as stored
    np.testing.assert_array_equal(read_gifti_mesh(tmp_path / "d.gii").faces, f)
    # a reference stored with another encoding: decoded and written anew
    text = (tmp_path / "a.gii").read_text()
    plain = base64.b64encode(f.astype("<i4").tobytes()).decode()
    faces_start = text.index("<DataArray", text.index("</DataArray>"))
    tail = text[faces_start:]
    tail = tail.replace('Encoding="GZipBase64Binary"', 'Encoding="Base64Binary"', 1)
    tail = re.sub(r"<Data>[^<]*</Data>", lambda _: f"<Data>{plain}</Data>", tail, count=1)
    (tmp_path / "e.gii").write_text(text[:faces_start] + tail)
    np.testing.assert_array_equal(read_gifti_mesh(tmp_path / "e.gii").faces, f)
    write_vertices_like(tmp_path / "e.gii", tmp_path / "g.gii", moved)
    g = read_gifti_mesh(tmp_path / "g.gii")
    np.testing.assert_array_equal(g.faces, f)
    np.testing.assert_array_equal(g.vertices, moved)
    with pytest.raises(ValueError):
        write_vertices_like(tmp_path / "a.gii", tmp_path / "h.gii", moved[:10])


def test_plan_only_topology_has_the_same_plan(native_library):
    from cat_surface_gpu_b200 import synthetic
    from cat_surface_gpu_b200.gifti import GiftiMesh
    from cat_surface_gpu_b200.surf2sphere import Surf2SphereTopology

    pts, tri = synthetic.folded_icosphere(4, seed=5, radius_mm=50.0)
    mesh = GiftiMesh(pts.astype(np.float32), tri.astype(np.int32))
    full, light = Surf2SphereTopology.from_mesh(mesh), Surf2SphereTopology.plan_only(mesh)
    for name in ("slot_off", "slot_tri", "order", "level_begin", "level_end"):
        np.testing.assert_array_equal(getattr(light.plan, name), getattr(full.plan, name))
    assert (light.plan.n_levels, light.plan.level_stride, light.plan.max_degree) == \
        (full.plan.n_levels, full.plan.level_stride, full.plan.max_degree)


def test_product_has_no_cpu_path():
    """Asking the product for a CPU device raises instead of falling back."""

    from cat_surface_gpu_b200.device import DeviceUnavailable, resolve_device

    with pytest.raises(DeviceUnavailable):
        resolve_device("cpu")


def test_gifti_reader_handles_wrapped_and_marked_up_payloads(tmp_path):
    """The reader parses the document without its payloads; payloads other writers wrap in
    lines or CDATA, and short ones, take the full parse and decode to the same arrays."""

    import re

    from cat_surface_gpu_b200.gifti import GiftiMesh, read_gifti_mesh, write_gifti_mesh

    from cat_surface_gpu_b200 import synthetic

    vertices, faces = synthetic.folded_icosphere(3, seed=11)
    write_gifti_mesh(tmp_path / "a.gii", GiftiMesh(vertices, faces))
    text = (tmp_path / "a.gii").read_text()
    wrapped = re.sub(r"<Data>([^<]*)</Data>",
                     lambda m: "<Data>" + "\n".join(m.group(1)[i:i + 76] for i in range(0, len(m.group(1)), 76))
                     + "\n</Data>", text)
    cdata = re.sub(r"<Data>([^<]*)</Data>", lambda m: "<Data><![CDATA[" + m.group(1) + "]]></Data>", text)
    for name, body in (("wrapped.gii", wrapped), ("cdata.gii", cdata)):
        (tmp_path / name).write_text(body)
        mesh = read_gifti_mesh(tmp_path / name)
        np.testing.assert_array_equal(mesh.vertices, np.asarray(vertices, dtype=np.float32))
        np.testing.assert_array_equal(mesh.faces, np.asarray(faces, dtype=np.int32))


def test_topology_caches_stay_bounded(native_library):
    """Many distinct meshes keep only the most recently used topology tables."""

    import torch

    from cat_surface_gpu_b200 import features, synthetic

    device = torch.device("cpu")
    first = None
    for seed in range(3 * features._CACHE_ENTRIES):
        vertices, faces = synthetic.folded_icosphere(1, seed=seed)
        faces = np.ascontiguousarray(faces, dtype=np.int32)[np.random.default_rng(seed).permutation(len(faces))]
        tables = features._topology(faces, vertices.shape[0], device)
        first = first if first is not None else (faces, tables)
        assert len(features._TOPOLOGY_CACHE) <= features._CACHE_ENTRIES
    again = features._topology(faces, vertices.shape[0], device)
    assert again is tables  # the latest mesh is still cached
    rebuilt = features._topology(first[0], vertices.shape[0], device)
    for a, b in zip(rebuilt[:4], first[1][:4]):  # the first one was evicted and is rebuilt the same
        assert torch.equal(a, b)
