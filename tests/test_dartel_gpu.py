"""GPU parity of the native DARTEL kernels (through the C ABI).

Element-wise operators must reproduce the reference's own outputs
(``tests/golden/dartel_golden.npz``, produced by the reference's torch path)
bit-for-bit in float64 and float32; whole steps and solves at the
configuration's 256 x 128 grid must equal the oracle restatement bit-for-bit.
Only reductions (the three diagnostics) and transcendental functions
(final warp) carry a tolerance, stated per test.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import GOLDEN
from oracle import dartel as od

pytestmark = pytest.mark.gpu

G = np.load(GOLDEN / "dartel_golden.npz")
TAGS = {"f64": torch.float64, "f32": torch.float32}
METRIC_RTOL = {"f64": 1e-11, "f32": 2e-5}


@pytest.fixture(scope="module")
def dg(native_library):
    from cat_surface_gpu_b200 import dartel_grid

    return dartel_grid


@pytest.fixture(scope="module")
def sw(native_library):
    from cat_surface_gpu_b200 import surface_warp

    return surface_warp


def g(tag, name):
    return G[f"{tag}/{name}"]


def cuda(x, tag):
    return torch.as_tensor(np.asarray(x)).to("cuda", TAGS[tag])


def host(t):
    return t.detach().cpu().numpy()


@pytest.mark.parametrize("tag", TAGS)
def test_maps_and_jacobians_bit_exact(dg, tag):
    dt = TAGS[tag]
    a, b, ja, jb, v = (cuda(g(tag, n), tag) for n in ("a", "b", "ja", "jb", "v"))
    np.testing.assert_array_equal(host(dg.composition(a, b, device="cuda", dtype=dt)), g(tag, "composition"))
    cm, cj = dg.composition_jacobian(a, ja, b, jb, device="cuda", dtype=dt)
    np.testing.assert_array_equal(host(cm), g(tag, "compj_map"))
    np.testing.assert_array_equal(host(cj), g(tag, "compj_jac"))
    np.testing.assert_array_equal(host(dg.jacobian_of_displacement(v, 0.25, device="cuda", dtype=dt)), g(tag, "jacdisp"))
    sm, sj = dg.smalldef_jac(v, -0.125, device="cuda", dtype=dt)
    np.testing.assert_array_equal(host(sm), g(tag, "smalldef_map"))
    np.testing.assert_array_equal(host(sj), g(tag, "smalldef_jac"))
    np.testing.assert_array_equal(host(dg.jac_div_smalldef(ja, v, 0.5, device="cuda", dtype=dt)), g(tag, "jacdiv"))
    for k in range(5):
        e, ej = dg.expdef(v, k, return_jacobian=True, device="cuda", dtype=dt)
        np.testing.assert_array_equal(host(e), g(tag, f"expdef_j_{k}_map"))
        np.testing.assert_array_equal(host(ej), g(tag, f"expdef_j_{k}_jac"))
        np.testing.assert_array_equal(host(dg.expdef(v, k, device="cuda", dtype=dt)), g(tag, f"expdef_{k}"))


@pytest.mark.parametrize("tag", TAGS)
def test_objective_and_squaring_bit_exact(dg, tag):
    dt = TAGS[tag]
    src, tgt, vel = (cuda(g(tag, n), tag) for n in ("src", "tgt", "vel"))
    t, j = dg.expdef(vel, 2, return_jacobian=True, device="cuda", dtype=dt)
    obj, rhs, hess = dg.initialise_objfun(src, tgt, t, j, device="cuda", dtype=dt)
    np.testing.assert_array_equal(host(rhs), g(tag, "objfun_rhs"))
    np.testing.assert_array_equal(host(hess), g(tag, "objfun_hess"))
    np.testing.assert_allclose(float(obj), float(g(tag, "objfun_obj")), rtol=METRIC_RTOL[tag])
    for k in range(6):
        for save in (False, True):
            sm, sj = dg.smalldef_jac(vel, -1.0 / 2 ** k, device="cuda", dtype=dt)
            res = dg.squaring_update(rhs, hess, sm, sj, k, save_transformation=save, return_scratch=True,
                                     device="cuda", dtype=dt)
            for name, value in zip(("b", "a", "map", "jac", "scratch"), res):
                np.testing.assert_array_equal(host(value), g(tag, f"sq_{k}_{int(save)}_{name}"), err_msg=f"{k} {save} {name}")


@pytest.mark.parametrize("tag", TAGS)
def test_regularisers_relax_resize_fmg_bit_exact(dg, tag):
    dt = TAGS[tag]
    vel, rhs, hpos, hess = (cuda(g(tag, n), tag) for n in ("vel", "objfun_rhs", "hpos", "objfun_hess"))
    params = (1.0, 1.0, 0.125, 0.05, 0.01)
    for rtype in (0, 1, 2):
        np.testing.assert_array_equal(host(dg.regularization_operator(vel, params, rtype, device="cuda", dtype=dt)),
                                      g(tag, f"reg_{rtype}"), err_msg=f"rtype {rtype}")
    np.testing.assert_array_equal(host(dg.apply_membrane_system(hpos, vel, params, device="cuda", dtype=dt)), g(tag, "apply"))
    np.testing.assert_array_equal(host(dg.relax_membrane(hpos, rhs, params, 3, vel, device="cuda", dtype=dt)), g(tag, "relax"))
    for name, (ny, nx) in (("r84", (4, 8)), ("r168", (16, 32)), ("r53", (2, 3)), ("r11", (1, 1)), ("r21", (1, 2))):
        out = dg.resize_field(hess, dg.GridSpec(nx=nx, ny=ny), device="cuda", dtype=dt)
        np.testing.assert_array_equal(host(out), g(tag, f"resize_{name}"), err_msg=name)
    out = dg.resize_field(cuda(g(tag, "resize_odd_in"), tag), dg.GridSpec(nx=4, ny=3), device="cuda", dtype=dt)
    np.testing.assert_array_equal(host(out), g(tag, "resize_odd"))
    fparams = (1.0, 1.0, 0.125, 0.0, 0.001)
    np.testing.assert_array_equal(host(dg.fmg2_membrane(hpos, rhs, fparams, 2, 2, None, device="cuda", dtype=dt)),
                                  g(tag, "fmg_none"))
    np.testing.assert_array_equal(host(dg.fmg2_membrane(hpos, rhs, fparams, 3, 3, vel, device="cuda", dtype=dt)),
                                  g(tag, "fmg_init"))


@pytest.mark.parametrize("tag", TAGS)
@pytest.mark.parametrize("code", (0, 1))
def test_dartel_step_matches_reference(dg, tag, code):
    dt = TAGS[tag]
    src, tgt, vel = (cuda(g(tag, n), tag) for n in ("src", "tgt", "vel"))
    for k in range(4):
        nv, m = dg.dartel_step(src, tgt, vel * 0.3, k=k, code=code, device="cuda", dtype=dt)
        np.testing.assert_array_equal(host(nv), g(tag, f"step_{code}_{k}_v"), err_msg=f"k={k}")
        np.testing.assert_allclose(host(m), g(tag, f"step_{code}_{k}_m"), rtol=METRIC_RTOL[tag])


@pytest.mark.parametrize("tag", TAGS)
@pytest.mark.parametrize("graph", (False, True))
def test_solve_matches_reference(sw, tag, graph):
    dt = TAGS[tag]
    res = sw.solve_dartel_maps(cuda(g(tag, "solve_src"), tag), cuda(g(tag, "solve_tgt"), tag), loop=2, its=2,
                               device="cuda", dtype=dt, cuda_graph=graph)
    np.testing.assert_array_equal(host(res.flow), g(tag, "solve_flow"))
    np.testing.assert_allclose(host(res.metrics), g(tag, "solve_metrics"), rtol=10 * METRIC_RTOL[tag])


@pytest.mark.parametrize("tag", TAGS)
def test_full_size_step_bit_exact_vs_oracle(dg, tag):
    """One dartel_step (k = 3, code 1) on the 256 x 128 sheet equals the oracle bit-for-bit."""

    from cat_surface_gpu_b200 import synthetic

    dtn = np.float64 if tag == "f64" else np.float32
    src = synthetic.smooth_sheet(128, 256, 1).astype(dtn)
    tgt = synthetic.smooth_sheet(128, 256, 2).astype(dtn)
    vel = (np.random.default_rng(5).normal(size=(2, 128, 256)) * 0.5).astype(dtn)
    want_v, want_m = od.dartel_step(src, tgt, vel, 3, params=(1.0, 1.0, 0.125, 0.0, 0.0), code=1)
    got_v, got_m = dg.dartel_step(cuda(src, tag), cuda(tgt, tag), cuda(vel, tag), k=3, device="cuda", dtype=TAGS[tag])
    np.testing.assert_array_equal(host(got_v), want_v)
    np.testing.assert_allclose(host(got_m), want_m, rtol=METRIC_RTOL[tag])


def test_batched_and_graph_solves_equal_single_solves(sw):
    """16 registrations in one batched launch sequence == 16 separate solves."""

    from cat_surface_gpu_b200 import synthetic

    ny, nx, batch = 32, 64, 16
    src = np.stack([synthetic.smooth_sheet(ny, nx, 10 + i) for i in range(batch)])
    tgt = np.stack([synthetic.smooth_sheet(ny, nx, 50 + i) for i in range(batch)])
    flows, _, metrics = sw.solve_dartel_batch(torch.as_tensor(src).cuda(), torch.as_tensor(tgt).cuda(), loop=3, its=2)
    for i in (0, 7, 15):
        single = sw.solve_dartel_maps(torch.as_tensor(src[i : i + 1]).cuda(), torch.as_tensor(tgt[i : i + 1]).cuda(),
                                      loop=3, its=2, assume_initial_nonzero=True)
        np.testing.assert_array_equal(host(flows[i]), host(single.flow))
        np.testing.assert_array_equal(host(metrics[i]), host(single.metrics[0]))
    eager = sw.solve_dartel_maps(torch.as_tensor(src[:2]).cuda(), torch.as_tensor(tgt[:2]).cuda(), loop=3, its=2)
    graphed = sw.solve_dartel_maps(torch.as_tensor(src[:2]).cuda(), torch.as_tensor(tgt[:2]).cuda(), loop=3, its=2,
                                   cuda_graph=True)
    graphed2 = sw.solve_dartel_maps(torch.as_tensor(src[2:4]).cuda(), torch.as_tensor(tgt[2:4]).cuda(), loop=3, its=2,
                                    cuda_graph=True)
    np.testing.assert_array_equal(host(eager.flow), host(graphed.flow))
    oracle_flow, _, _ = od.solve_dartel_maps(src[2:4], tgt[2:4], loop=3, its=2)
    np.testing.assert_array_equal(host(graphed2.flow), oracle_flow)


def test_registration_batch_equals_one_at_a_time(sw):
    """R registrations x 2 step maps in one batched solve == R solve_dartel_maps calls (eager and graphed)."""

    from cat_surface_gpu_b200 import synthetic

    ny, nx, regs, steps = 32, 64, 5, 2
    src = np.stack([[synthetic.smooth_sheet(ny, nx, 100 + 2 * r + s) for s in range(steps)] for r in range(regs)])
    tgt = np.stack([[synthetic.smooth_sheet(ny, nx, 300 + 2 * r + s) for s in range(steps)] for r in range(regs)])
    s_dev, t_dev = torch.as_tensor(src).cuda(), torch.as_tensor(tgt).cuda()
    for graph in (False, True):
        flows, metrics = sw.solve_dartel_registrations(s_dev, t_dev, loop=3, its=2, cuda_graph=graph)
        assert tuple(flows.shape) == (regs, 2, ny, nx) and tuple(metrics.shape) == (regs, steps, 6, 3)
        for r in range(regs):
            one = sw.solve_dartel_maps(s_dev[r], t_dev[r], loop=3, its=2, cuda_graph=graph)
            np.testing.assert_array_equal(host(flows[r]), host(one.flow))
            np.testing.assert_array_equal(host(metrics[r]), host(one.metrics))


@pytest.mark.parametrize("tag", TAGS)
def test_final_warp_and_average(sw, tag):
    flow = cuda(g(tag, "solve_flow"), tag)
    pts = g(tag, "warp_points")
    out = sw.apply_flow_to_sphere(torch.as_tensor(pts).cuda(), flow, unit_sphere_vertices=torch.as_tensor(pts).cuda(),
                                  inverse=True, device="cuda", dtype=TAGS[tag])
    np.testing.assert_allclose(host(out), g(tag, "warp_out"), rtol=0, atol=1e-12 if tag == "f64" else 2e-6)
    avg = sw.average_xz_surfaces(torch.as_tensor(G["avg_x"]).cuda(), torch.as_tensor(G["avg_z"]).cuda(), device="cuda")
    np.testing.assert_allclose(host(avg), G["avg_out"], rtol=0, atol=1e-6)


def test_dartel_argument_errors(dg):
    with pytest.raises(ValueError):
        dg.relax_membrane(torch.zeros(3, 3, 5, device="cuda", dtype=torch.float64),
                          torch.zeros(2, 3, 5, device="cuda", dtype=torch.float64), (1, 1, 0.1, 0, 0), 2)
    with pytest.raises(ValueError):
        dg.composition(torch.zeros(3, 4, 4, device="cuda"), torch.zeros(3, 4, 4, device="cuda"), device="cuda")
    with pytest.raises(ValueError):
        dg.regularization_operator(torch.zeros(2, 4, 4, device="cuda", dtype=torch.float64), (1, 1, 0.1, 0, 0), rtype=3)
    with pytest.raises(dg.DeviceUnavailable):
        dg.expdef(torch.zeros(2, 4, 4), 2, device="cpu")
