"""The DARTEL oracle is pinned to the reference's own outputs (golden vectors).

``tests/golden/dartel_golden.npz`` was produced by running the reference
package's torch CPU path (``make_dartel_golden.py``).  Element-wise operators
must match bit-for-bit (same operation order, one rounding per operation);
quantities that go through a reduction or a transcendental function match to
1e-12 relative (float64) / 1e-5 (float32).
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import dartel as od

G = np.load(GOLDEN / "dartel_golden.npz")
TAGS = ("f64", "f32")


def g(tag, name):
    return G[f"{tag}/{name}"]


@pytest.mark.parametrize("tag", TAGS)
def test_composition_and_jacobians_bit_exact(tag):
    a, b, ja, jb, v = (g(tag, n) for n in ("a", "b", "ja", "jb", "v"))
    np.testing.assert_array_equal(od.composition(a, b), g(tag, "composition"))
    cm, cj = od.composition_jacobian(a, ja, b, jb)
    np.testing.assert_array_equal(cm, g(tag, "compj_map"))
    np.testing.assert_array_equal(cj, g(tag, "compj_jac"))
    np.testing.assert_array_equal(od.jacobian_of_displacement(v, 0.25), g(tag, "jacdisp"))
    sm, sj = od.smalldef_jac(v, -0.125)
    np.testing.assert_array_equal(sm, g(tag, "smalldef_map"))
    np.testing.assert_array_equal(sj, g(tag, "smalldef_jac"))
    np.testing.assert_array_equal(od.jac_div_smalldef(ja, v, 0.5), g(tag, "jacdiv"))


@pytest.mark.parametrize("tag", TAGS)
@pytest.mark.parametrize("k", range(5))
def test_expdef_bit_exact(tag, k):
    v = g(tag, "v")
    e, ej = od.expdef(v, k, return_jacobian=True)
    np.testing.assert_array_equal(e, g(tag, f"expdef_j_{k}_map"))
    np.testing.assert_array_equal(ej, g(tag, f"expdef_j_{k}_jac"))
    np.testing.assert_array_equal(od.expdef(v, k), g(tag, f"expdef_{k}"))


@pytest.mark.parametrize("tag", TAGS)
def test_objective_and_squaring(tag):
    src, tgt, vel = g(tag, "src"), g(tag, "tgt"), g(tag, "vel")
    t, j = od.expdef(vel, 2, return_jacobian=True)
    obj, rhs, hess = od.initialise_objfun(src, tgt, t, j)
    np.testing.assert_array_equal(rhs, g(tag, "objfun_rhs"))
    np.testing.assert_array_equal(hess, g(tag, "objfun_hess"))
    np.testing.assert_allclose(obj, g(tag, "objfun_obj"), rtol=1e-12 if tag == "f64" else 1e-5)
    for k in range(6):
        for save in (False, True):
            sm, sj = od.smalldef_jac(vel, -1.0 / 2 ** k)
            res = od.squaring_update(rhs, hess, sm, sj, k, save_transformation=save)
            for name, value in zip(("b", "a", "map", "jac", "scratch"), res):
                np.testing.assert_array_equal(value, g(tag, f"sq_{k}_{int(save)}_{name}"), err_msg=f"{k} {save} {name}")


@pytest.mark.parametrize("tag", TAGS)
def test_regularisers_relax_resize(tag):
    vel, rhs, hpos = g(tag, "vel"), g(tag, "objfun_rhs"), g(tag, "hpos")
    params = (1.0, 1.0, 0.125, 0.05, 0.01)
    for rtype in (0, 1, 2):
        np.testing.assert_array_equal(od.regularization_operator(vel, params, rtype), g(tag, f"reg_{rtype}"))
    np.testing.assert_array_equal(od.apply_membrane_system(hpos, vel, params), g(tag, "apply"))
    np.testing.assert_array_equal(od.relax_membrane(hpos, rhs, params, 3, vel), g(tag, "relax"))
    np.testing.assert_array_equal(
        od.relax_membrane(hpos[:, :3, :5].copy(), rhs[:, :3, :5].copy(), params, 2, None), g(tag, "relax_odd")
    )
    hess = g(tag, "objfun_hess")
    for name, (ny, nx) in (("r84", (4, 8)), ("r168", (16, 32)), ("r53", (2, 3)), ("r11", (1, 1)), ("r21", (1, 2))):
        np.testing.assert_array_equal(od.resize_field(hess, nx, ny), g(tag, f"resize_{name}"), err_msg=name)
    np.testing.assert_array_equal(od.resize_field(g(tag, "resize_odd_in"), 4, 3), g(tag, "resize_odd"))


@pytest.mark.parametrize("tag", TAGS)
def test_multigrid_bit_exact(tag):
    rhs, hpos, vel = g(tag, "objfun_rhs"), g(tag, "hpos"), g(tag, "vel")
    fparams = (1.0, 1.0, 0.125, 0.0, 0.001)
    np.testing.assert_array_equal(od.fmg2_membrane(hpos, rhs, fparams, 2, 2, None), g(tag, "fmg_none"))
    np.testing.assert_array_equal(od.fmg2_membrane(hpos, rhs, fparams, 3, 3, vel), g(tag, "fmg_init"))


@pytest.mark.parametrize("tag", TAGS)
@pytest.mark.parametrize("code", (0, 1))
def test_dartel_step(tag, code):
    src, tgt, vel = g(tag, "src"), g(tag, "tgt"), g(tag, "vel")
    for k in range(4):
        nv, m = od.dartel_step(src, tgt, vel * vel.dtype.type(0.3), k, code=code)
        np.testing.assert_array_equal(nv, g(tag, f"step_{code}_{k}_v"), err_msg=f"k={k}")
        np.testing.assert_allclose(m, g(tag, f"step_{code}_{k}_m"), rtol=1e-11 if tag == "f64" else 2e-5)


@pytest.mark.parametrize("tag", TAGS)
def test_solve_and_warp(tag):
    flow, metrics, _ = od.solve_dartel_maps(g(tag, "solve_src"), g(tag, "solve_tgt"), loop=2, its=2)
    np.testing.assert_array_equal(flow, g(tag, "solve_flow"))
    np.testing.assert_allclose(metrics, g(tag, "solve_metrics"), rtol=1e-10 if tag == "f64" else 1e-4)
    warped = od.apply_flow_to_sphere(g(tag, "warp_points"), flow)
    np.testing.assert_allclose(warped, g(tag, "warp_out"), rtol=0, atol=1e-12 if tag == "f64" else 2e-6)


def test_average_and_schedule():
    np.testing.assert_allclose(od.average_xz_surfaces(G["avg_x"], G["avg_z"]), G["avg_out"], rtol=0, atol=1e-6)
    np.testing.assert_allclose(np.asarray(od.default_dartel_parameters(6)), G["mu_schedule"], rtol=0, atol=0)
    # the reference's own known answer: mu 0.125 x 4 then 0.1 x 2 (test_surface_stencil.py:145-150)
    assert [p[2] for p in od.default_dartel_parameters(6)] == [0.125] * 4 + [0.1] * 2
