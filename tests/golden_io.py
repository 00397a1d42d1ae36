"""Loading helpers for the committed golden fixtures."""
from pathlib import Path

import numpy as np

from stargaze_b200.pathtracer import RAY_DTYPE

GOLDEN = Path(__file__).resolve().parent / "golden"
RAY_SCENES = ["transport", "spheres_256", "rings_1080p", "shadow_ring", "terrain", "vegetation"]
IMAGE_NAMES = ["spheres_64", "rings_96x54", "terrain_96x54", "terrain_air_96x54", "styles_96x32",
               "terrain_alpine_96x54", "terrain_dunes_96x54", "terrain_basalt_96x54",
               "terrain_vegetation_96x54", "mottled_96x54"]


def load_rays(name: str) -> dict:
    z = np.load(GOLDEN / f"rays_{name}.npz")
    d = dict(z)
    d["rays"] = np.ascontiguousarray(d["rays"]).view(RAY_DTYPE).reshape(-1)
    d["vis_rays"] = np.ascontiguousarray(d["vis_rays"]).view(RAY_DTYPE).reshape(-1)
    return d


def load_image(name: str) -> np.ndarray:
    return np.load(GOLDEN / f"image_{name}.npz")["image"]


def relative_rmse(x: np.ndarray, reference: np.ndarray) -> float:
    """sqrt(sum (x - y)^2 / sum y^2) over RGB, W excluded
    (scripts/benchmark.py:219-232 of the reference)."""
    a = x[..., :3].astype(np.float64)
    b = reference[..., :3].astype(np.float64)
    den = float((b * b).sum())
    return float(np.sqrt(((a - b) ** 2).sum() / den)) if den > 0 else float(np.sqrt(((a - b) ** 2).sum()))
