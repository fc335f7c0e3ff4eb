"""Generate DARTEL / warp golden vectors by running the reference package on CPU.

Runs in the development container only: it imports ``cat_surface_gpu`` from
the reference checkout (``$CAT_SURFACE_REFERENCE/src``) and evaluates its torch CPU
path on seeded small grids.  The committed ``dartel_golden.npz`` holds every
input and output, so tests never need the reference at run time.

Usage: ``python tests/golden/make_dartel_golden.py``
"""

from __future__ import annotations

import os
from pathlib import Path
import sys

import numpy as np

os.environ.setdefault("PYTHONDONTWRITEBYTECODE", "1")
sys.dont_write_bytecode = True
sys.path.insert(0, str(Path(__file__).resolve().parent))
from _reference import use_reference_package  # noqa: E402

REFERENCE_SRC = use_reference_package()

import torch  # noqa: E402

from cat_surface_gpu import dartel_grid as dg  # noqa: E402
from cat_surface_gpu import surface_warp as sw  # noqa: E402
from cat_surface_gpu import gpu_pipeline as gp  # noqa: E402

OUT = Path(__file__).resolve().parent / "dartel_golden.npz"


def smooth(ny, nx, seed, dtype):
    rng = np.random.default_rng(seed)
    y = (np.arange(ny) + 0.5) / ny
    x = (np.arange(nx) + 0.5) / nx
    yy, xx = np.meshgrid(y, x, indexing="ij")
    total = np.zeros((ny, nx))
    for _ in range(6):
        kx, ky = rng.integers(1, 4, size=2)
        total += rng.normal() * np.cos(2 * np.pi * kx * xx + rng.uniform(0, 6)) * np.sin(np.pi * ky * yy + rng.uniform(0, 3))
    total -= total.min()
    total /= total.max()
    return total.astype(dtype)


def main() -> int:
    out: dict[str, np.ndarray] = {}
    cpu = torch.device("cpu")
    for tag, dtype, tdtype in (("f64", np.float64, torch.float64), ("f32", np.float32, torch.float32)):
        rng = np.random.default_rng(7 if tag == "f64" else 8)
        ny, nx = 7, 9
        spec = dg.GridSpec(nx=nx, ny=ny)
        ident = dg.make_identity_map(spec, device=cpu, dtype=tdtype)
        a = (ident + torch.as_tensor(rng.normal(size=(2, ny, nx)) * 1.7, dtype=tdtype)).contiguous()
        b = (ident + torch.as_tensor(rng.normal(size=(2, ny, nx)) * 0.8, dtype=tdtype)).contiguous()
        ja = torch.as_tensor(rng.normal(size=(4, ny, nx)) * 0.3 + np.array([1, 0, 0, 1])[:, None, None], dtype=tdtype)
        jb = torch.as_tensor(rng.normal(size=(4, ny, nx)) * 0.3 + np.array([1, 0, 0, 1])[:, None, None], dtype=tdtype)
        v = torch.as_tensor(rng.normal(size=(2, ny, nx)) * 0.6, dtype=tdtype)
        out[f"{tag}/a"], out[f"{tag}/b"], out[f"{tag}/ja"], out[f"{tag}/jb"], out[f"{tag}/v"] = (
            t.numpy() for t in (a, b, ja, jb, v)
        )
        out[f"{tag}/composition"] = dg.composition(a, b, device=cpu, dtype=tdtype).numpy()
        cm, cj = dg.composition_jacobian(a, ja, b, jb, device=cpu, dtype=tdtype)
        out[f"{tag}/compj_map"], out[f"{tag}/compj_jac"] = cm.numpy(), cj.numpy()
        out[f"{tag}/jacdisp"] = dg.jacobian_of_displacement(v, 0.25, device=cpu, dtype=tdtype).numpy()
        sm, sj = dg.smalldef_jac(v, -0.125, device=cpu, dtype=tdtype)
        out[f"{tag}/smalldef_map"], out[f"{tag}/smalldef_jac"] = sm.numpy(), sj.numpy()
        out[f"{tag}/jacdiv"] = dg.jac_div_smalldef(ja, v, 0.5, device=cpu, dtype=tdtype).numpy()
        for k in range(5):
            e, ej = dg.expdef(v, k, return_jacobian=True, device=cpu, dtype=tdtype)
            out[f"{tag}/expdef_j_{k}_map"], out[f"{tag}/expdef_j_{k}_jac"] = e.numpy(), ej.numpy()
            out[f"{tag}/expdef_{k}"] = dg.expdef(v, k, device=cpu, dtype=tdtype).numpy()

        # objective / squaring on a 16 x 8 grid
        ny2, nx2 = 8, 16
        spec2 = dg.GridSpec(nx=nx2, ny=ny2)
        src = torch.as_tensor(smooth(ny2, nx2, 1, dtype))
        tgt = torch.as_tensor(smooth(ny2, nx2, 2, dtype))
        vel = torch.as_tensor(rng.normal(size=(2, ny2, nx2)) * 0.8, dtype=tdtype)
        out[f"{tag}/src"], out[f"{tag}/tgt"], out[f"{tag}/vel"] = src.numpy(), tgt.numpy(), vel.numpy()
        t, j = dg.expdef(vel, 2, return_jacobian=True, device=cpu, dtype=tdtype)
        obj, rhs, hess = dg.initialise_objfun(src, tgt, t, j, device=cpu, dtype=tdtype)
        out[f"{tag}/objfun_obj"], out[f"{tag}/objfun_rhs"], out[f"{tag}/objfun_hess"] = obj.numpy(), rhs.numpy(), hess.numpy()
        for k in range(6):
            for save in (False, True):
                sm2, sj2 = dg.smalldef_jac(vel, -1.0 / 2 ** k, device=cpu, dtype=tdtype)
                res = dg.squaring_update(rhs, hess, sm2, sj2, k, save_transformation=save, return_scratch=True,
                                         device=cpu, dtype=tdtype, optimized=True, kernel="torch")
                for name, value in zip(("b", "a", "map", "jac", "scratch"), res):
                    out[f"{tag}/sq_{k}_{int(save)}_{name}"] = value.numpy()
        params = (1.0, 1.0, 0.125, 0.05, 0.01)
        for rtype in (0, 1, 2):
            out[f"{tag}/reg_{rtype}"] = dg.regularization_operator(vel, params, rtype, device=cpu, dtype=tdtype).numpy()
        hpos = torch.abs(hess) + 0.01
        hpos[2] = hess[2] * 0.1
        out[f"{tag}/hpos"] = hpos.numpy()
        out[f"{tag}/apply"] = dg.apply_membrane_system(hpos, vel, params, kernel="torch", device=cpu, dtype=tdtype).numpy()
        out[f"{tag}/relax"] = dg.relax_membrane(hpos, rhs, params, 3, vel, kernel="torch", device=cpu, dtype=tdtype).numpy()
        # odd nx: the reference's sequential scalar red-black path
        h_odd = hpos[:, :3, :5].contiguous()
        r_odd = rhs[:, :3, :5].contiguous()
        out[f"{tag}/relax_odd"] = dg.relax_membrane(h_odd, r_odd, params, 2, None, kernel="torch", device=cpu, dtype=tdtype).numpy()
        for name, shape in (("r84", (4, 8)), ("r168", (16, 32)), ("r53", (2, 3)), ("r11", (1, 1)), ("r21", (1, 2))):
            out[f"{tag}/resize_{name}"] = dg.resize_field(hess, dg.GridSpec(nx=shape[1], ny=shape[0]), kernel="torch",
                                                           device=cpu, dtype=tdtype).numpy()
        out[f"{tag}/resize_odd_in"] = rhs[:, :5, :7].contiguous().numpy()
        out[f"{tag}/resize_odd"] = dg.resize_field(rhs[:, :5, :7].contiguous(), dg.GridSpec(nx=4, ny=3), kernel="torch",
                                                   device=cpu, dtype=tdtype).numpy()
        fparams = (1.0, 1.0, 0.125, 0.0, 0.001)
        out[f"{tag}/fmg_none"] = dg.fmg2_membrane(hpos, rhs, fparams, 2, 2, None, kernel="torch", device=cpu, dtype=tdtype).numpy()
        out[f"{tag}/fmg_init"] = dg.fmg2_membrane(hpos, rhs, fparams, 3, 3, vel, kernel="torch", device=cpu, dtype=tdtype).numpy()
        for code in (0, 1):
            for k in range(4):
                nv, m = dg.dartel_step(src, tgt, vel * 0.3, k=k, params=(1.0, 1.0, 0.125, 0.0, 0.0), code=code,
                                       kernel="torch", device=cpu, dtype=tdtype)
                out[f"{tag}/step_{code}_{k}_v"], out[f"{tag}/step_{code}_{k}_m"] = nv.numpy(), m.numpy()
        maps_s = torch.stack((src, torch.as_tensor(smooth(ny2, nx2, 3, dtype))))
        maps_t = torch.stack((tgt, torch.as_tensor(smooth(ny2, nx2, 4, dtype))))
        res = sw.solve_dartel_maps(maps_s, maps_t, loop=2, its=2, kernel="torch", device=cpu, dtype=tdtype)
        out[f"{tag}/solve_src"], out[f"{tag}/solve_tgt"] = maps_s.numpy(), maps_t.numpy()
        out[f"{tag}/solve_flow"], out[f"{tag}/solve_metrics"] = res.flow.numpy(), res.metrics.numpy()
        pts = rng.normal(size=(400, 3))
        pts /= np.linalg.norm(pts, axis=1, keepdims=True)
        pts = pts.astype(np.float32)
        out[f"{tag}/warp_points"] = pts
        out[f"{tag}/warp_out"] = sw.apply_flow_to_sphere(torch.as_tensor(pts), res.flow, unit_sphere_vertices=torch.as_tensor(pts),
                                                        inverse=True, device=cpu, dtype=tdtype).numpy()
    rng = np.random.default_rng(3)
    xs = rng.normal(size=(300, 3)); xs /= np.linalg.norm(xs, axis=1, keepdims=True)
    zs = rng.normal(size=(300, 3)); zs /= np.linalg.norm(zs, axis=1, keepdims=True)
    out["avg_x"], out["avg_z"] = xs, zs
    out["avg_out"] = gp._average_xz_surfaces(torch.as_tensor(xs), torch.as_tensor(zs), device=cpu).numpy()
    out["mu_schedule"] = np.asarray(sw.default_dartel_parameters(6))
    np.savez_compressed(OUT, **out)
    print(OUT, len(out), "arrays")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
