"""kerrray_b200: KerrRay's per-ray ray-tracing hot path on NVIDIA B200 (sm_100a).

A drop-in ``cuda`` backend for KerrRay's ``Backend`` protocol plus batched (many images in one
persistent launch) entry points. The compute runs in ``libkerrray_cuda.so`` (hand-written CUDA
C++ behind the C ABI of ``include/kerrray_cuda.h``); this package is the host side.
"""

from kerrray_b200._lib import BackendUnavailable
from kerrray_b200.adjoint import (
    LensingFunction,
    LensingResult,
    edge_distant_rays,
    fit_spin_inclination,
    lensing_map,
    magnification,
)
from kerrray_b200.autotune import autotune, list_variants
from kerrray_b200.backends import (
    BACKEND_NAMES,
    Backend,
    CudaBackend,
    available_backends,
    get_backend,
    register_with_kerrray,
)
from kerrray_b200.bisect import EdgeCase, bisect_edge, bisect_edges, edge_options, edge_study
from kerrray_b200.boundary import (
    analytic_boundary,
    boundary_error,
    extract_boundary_from_mask,
    finite_distance_scale,
    mask_edge_error,
    polygon_centroid,
    polygon_radii,
)
from kerrray_b200.camera import Camera, initial_states, initial_states_at
from kerrray_b200.orbits import BardeenCurve, critical_impact_parameters, shadow_curve
from kerrray_b200.rays import trace_rays
from kerrray_b200.renderer import DiskImage, DiskModel, load_disk_image_arrays, render_disk, save_disk_image
from kerrray_b200.shadow import FAILURE_STATES, ShadowImage, compute_shadow, shadow_mask_int8, state_counts
from kerrray_b200.sweep import (
    RETRACE_CRITICAL,
    RETRACE_CRITICAL_NEAR,
    RETRACE_EDGE,
    DeviceSweep,
    ImageSpec,
    LaunchConfig,
    SweepResult,
    analytic_classes,
    direction_angle,
    escape_directions,
    trig_eval,
    order_by_cost,
    trace_images,
)
from kerrray_b200.validation import (
    critical_impacts,
    equatorial_photon,
    photon_from_constants,
    photon_sphere,
    tangential_photon,
    winding_rate_prediction,
    winding_rates,
)
from kerrray_b200.types import (
    BatchResult,
    EventOptions,
    IntegratorOptions,
    Spacetime,
    TerminationOptions,
    TerminationState,
    max_attempts,
    outer_horizon,
)

__all__ = [
    "LensingFunction", "LensingResult", "edge_distant_rays", "fit_spin_inclination", "lensing_map", "magnification",
    "critical_impacts", "equatorial_photon", "photon_from_constants", "photon_sphere", "tangential_photon",
    "winding_rate_prediction", "winding_rates",
    "EdgeCase", "analytic_boundary", "bisect_edge", "bisect_edges", "boundary_error", "critical_impact_parameters",
    "edge_options", "edge_study", "extract_boundary_from_mask", "finite_distance_scale", "polygon_centroid",
    "polygon_radii", "shadow_curve", "mask_edge_error", "BardeenCurve",
    "BACKEND_NAMES", "Backend", "BackendUnavailable", "BatchResult", "Camera", "CudaBackend", "DeviceSweep",
    "EventOptions", "FAILURE_STATES", "ImageSpec", "IntegratorOptions", "LaunchConfig", "ShadowImage", "Spacetime",
    "SweepResult", "TerminationOptions", "TerminationState", "autotune", "available_backends", "compute_shadow",
    "get_backend", "initial_states", "initial_states_at", "list_variants", "max_attempts", "order_by_cost",
    "outer_horizon", "register_with_kerrray", "shadow_mask_int8", "state_counts", "trace_images", "trace_rays",
    "RETRACE_CRITICAL", "RETRACE_CRITICAL_NEAR", "RETRACE_EDGE", "analytic_classes", "direction_angle", "escape_directions", "trig_eval",
    "DiskImage", "DiskModel", "load_disk_image_arrays", "render_disk", "save_disk_image",
]
