"""B200-native CAT-Surface hot paths with the reference's public API.

Same public names as the reference package (``src/cat_surface_gpu/__init__.py``):
Surf2Sphere area smoothing, DARTEL operators and solves, rotation search,
stencils and the end-to-end SurfWarp pipeline.  Numerics run in native
sm_100a kernels (``libcatsurf_b200.so``); there is no CPU fallback.
Submodules import lazily so that ``import cat_surface_gpu_b200`` works on a
machine without a GPU.
"""

from __future__ import annotations

import importlib

_EXPORTS = {
    "dartel_grid": ["DeviceUnavailable", "GridSpec", "composition", "composition_jacobian", "dartel_step", "expdef",
                    "fmg2_membrane", "from_c_layout", "initialise_objfun", "jacobian_of_displacement",
                    "jac_div_smalldef", "make_identity_map", "apply_membrane_system", "relax_membrane",
                    "regularization_operator", "resolve_device", "resize_field", "sample_field", "smalldef_jac",
                    "squaring_update", "to_c_layout"],
    "surface_stencil": ["SurfaceStencil", "SurfaceStencilDevice", "build_surface_stencil"],
    "surface_rotation": ["RotationCostInputs", "RotationGridIndex", "RotationGridIndexDevice", "RotationSearchResult",
                         "official_seed_grid_angles", "batched_costs"],
    "rotation_pipeline": ["RotationPipeline", "read_rotation_points", "read_rotation_values", "run_rotation_pipeline",
                          "run_rotation_pipeline_from_files"],
    "surface_warp": ["DartelSolveResult", "apply_flow_to_sphere", "apply_flow_to_stenciled_sphere",
                     "clear_dartel_cuda_graph_cache", "default_dartel_parameters", "prepare_dartel_cuda_graph",
                     "solve_dartel_from_surfaces", "solve_dartel_maps", "solve_dartel_batch", "solve_dartel_registrations",
                     "average_xz_surfaces"],
    "gpu_pipeline": ["CatSurfaceGpuResult", "run_cat_surface_gpu_pipeline"],
    "gifti": ["GiftiMesh", "read_gifti_mesh", "write_gifti_mesh"],
    "surf2sphere": ["CatSurf2SphereGpuResult", "Surf2SphereTopology", "convert_ellipsoid_to_sphere_with_surface_area",
                    "run_areal_smoothing_cuda", "run_cat_surf2sphere_gpu", "run_surf2sphere_preprocess_cuda",
                    "surface_area"],
}
_WHERE = {name: module for module, names in _EXPORTS.items() for name in names}
__all__ = sorted(_WHERE)


def __getattr__(name: str):
    module = _WHERE.get(name)
    if module is None:
        raise AttributeError(f"module 'cat_surface_gpu_b200' has no attribute {name!r}")
    return getattr(importlib.import_module(f".{module}", __name__), name)
