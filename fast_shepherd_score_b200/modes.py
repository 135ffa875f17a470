"""Alignment modes: result attribute names and per-mode defaults.

The tables restate shepherd_score/accel/_modes.py:18-61 (they must be identical: results are
written onto MoleculePair objects under these names, and the per-mode seed/step defaults
decide what a call without explicit ``num_repeats``/``max_num_steps`` runs).  ``vol_pharm``
(shape + directional pharmacophore with one shared pose) is this backend's addition.
"""
from __future__ import annotations

MODE_ATTRS = {
    "vol": ("transform_vol_noH", "sim_aligned_vol_noH"),
    "vol_esp": ("transform_vol_esp_noH", "sim_aligned_vol_esp_noH"),
    "surf": ("transform_surf", "sim_aligned_surf"),
    "surf_esp": ("transform_surf_esp", "sim_aligned_surf_esp"),
    "vol_and_surf_esp": ("transform_vol_and_surf_esp", "sim_aligned_vol_and_surf_esp"),
    "pharm": ("transform_pharm", "sim_aligned_pharm"),
    "vol_color": ("transform_vol_color", "sim_aligned_vol_color"),
    "vol_pharm": ("transform_vol_pharm", "sim_aligned_vol_pharm"),
}
CANONICAL_MODES = tuple(MODE_ATTRS)
LEGACY_MODE_ALIASES = {"esp": "surf_esp", "esp_combo": "vol_and_surf_esp"}
MODE_SEEDS = {"vol": 10, "surf": 8, "surf_esp": 8, "vol_esp": 16, "vol_and_surf_esp": 8,
              "pharm": 32, "vol_color": 16, "vol_pharm": 16}
MODE_STEPS = {"vol": 30, "surf": 40, "surf_esp": 40, "vol_esp": 50, "vol_and_surf_esp": 60,
              "pharm": 50, "vol_color": 40, "vol_pharm": 40}
# modes the CUDA backend implements
CUDA_MODES = ("vol", "vol_esp", "surf", "surf_esp", "vol_and_surf_esp", "pharm", "vol_color",
              "vol_pharm")


def canonical(mode: str) -> str:
    """Resolve a (possibly legacy) mode name; unknown names pass through."""
    return LEGACY_MODE_ALIASES.get(mode, mode)


def seeds_for(mode: str) -> int:
    return MODE_SEEDS.get(canonical(mode), 50)


def steps_for(mode: str) -> int:
    return MODE_STEPS.get(canonical(mode), 50)
