"""taichirtm_b200 -- B200-native (sm_100a) 2-D elastic reverse-time migration.

Drop-in for TaichiRTM's public API (src/__init__.py:24-55): the same classes
and functions, with the propagation done by hand-written CUDA in
``lib/librtm_b200.so`` (C ABI: include/rtm_b200.h)."""
from .backward_modeling import BackwardModeling
from .forward_modeling import ForwardModeling
from .imaging import (
    compute_display_limits,
    create_visualization_data,
    load_rtm_results,
    prepare_image_data,
    save_stacked_results,
    stack_rtm_images,
)
from .rtm import ReverseTimeMigration, init_taichi, reset_taichi

__version__ = "2.0.0"

__all__ = [
    "ReverseTimeMigration",
    "init_taichi",
    "reset_taichi",
    "ForwardModeling",
    "BackwardModeling",
    "load_rtm_results",
    "stack_rtm_images",
    "compute_display_limits",
    "prepare_image_data",
    "create_visualization_data",
    "save_stacked_results",
]
