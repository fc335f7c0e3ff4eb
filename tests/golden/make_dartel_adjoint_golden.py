"""Generate the reference's DARTEL data-term gradient on CPU, for the adjoint tests.

Development container only (imports ``cat_surface_gpu`` from the reference
checkout).  For seeded 64 x 32 float64 sheets S, T and a smooth velocity v,
and k in (0, 3, 7), evaluates with the reference's own torch CPU functions:

* ``objective``  -- initialise_objfun's 1/2 sum (S(exp v) - T)^2 at exp(v) = expdef(v, k);
* ``gradient``   -- its Gauss-Newton gradient pulled back through squaring_update
                    and scaled by 2^-k, as dartel_step forms it before the
                    regulariser (dartel_grid.py:1420-1616, code 0).

Writes ``dartel_adjoint_golden.npz``.  Usage:
``python tests/golden/make_dartel_adjoint_golden.py``
"""

from __future__ import annotations

import os
from pathlib import Path
import sys

import numpy as np

os.environ.setdefault("PYTHONDONTWRITEBYTECODE", "1")
sys.dont_write_bytecode = True
HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))
sys.path.insert(0, str(HERE))
from _reference import use_reference_package  # noqa: E402

use_reference_package()

import torch  # noqa: E402

from cat_surface_gpu import dartel_grid as dg  # noqa: E402

from cat_surface_gpu_b200 import synthetic  # noqa: E402

KS = (0, 3, 7)
NY, NX = 32, 64


def inputs():
    source = synthetic.smooth_sheet(NY, NX, 21).astype(np.float64)
    target = synthetic.smooth_sheet(NY, NX, 22).astype(np.float64)
    velocity = np.stack([synthetic.smooth_sheet(NY, NX, 23 + c) - 0.5 for c in range(2)]) * 3.0
    return source, target, velocity


def reference_gradient(source, target, velocity, k):
    cpu = torch.device("cpu")
    v = torch.as_tensor(velocity)
    s = 1.0 / 2 ** k
    t, jac = dg.expdef(v, k, return_jacobian=True, device=cpu)
    jac = dg.jac_div_smalldef(jac, v, s, device=cpu)
    objective, rhs, hess = dg.initialise_objfun(torch.as_tensor(source), torch.as_tensor(target), t, jac, device=cpu)
    t2, j2 = dg.smalldef_jac(v, -s, device=cpu)
    rhs, _, _, _ = dg.squaring_update(rhs, hess, t2, j2, k, device=cpu)
    return float(objective), (rhs * s).numpy()


def main() -> int:
    source, target, velocity = inputs()
    out = {"source": source, "target": target, "velocity": velocity, "ks": np.asarray(KS)}
    for k in KS:
        objective, gradient = reference_gradient(source, target, velocity, k)
        out[f"objective_{k}"] = np.float64(objective)
        out[f"gradient_{k}"] = gradient
    np.savez_compressed(HERE / "dartel_adjoint_golden.npz", **out)
    print("wrote", HERE / "dartel_adjoint_golden.npz")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
