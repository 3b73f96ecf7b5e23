"""Mesh loading (drop-in for src/mesh/loader.py:11-108).

Same file layout, 1-based-to-0-based conversion, validation and errors as the
reference.  Addition: ``mesh_dir=None`` generates the reference's structured
meshes instead of reading files (bit-identical to data/mesh/richards/p*.csv,
t*.csv, p_3D/t_3D and data/mesh/nitrogen/*); unit-square cases
(NitrogenTest, VGDirichlet) use side length 1.
"""
import io
import zipfile
from pathlib import Path
from typing import Any, Dict, Optional, Tuple

import numpy as np

from wspm_b200 import mesh as gen


def _read_csv(path: Path, dtype):
    if path.suffix == ".zip":
        with zipfile.ZipFile(path) as z:
            name = z.namelist()[0]
            return np.loadtxt(io.StringIO(z.read(name).decode()), delimiter=",", dtype=dtype, ndmin=2)
    return np.loadtxt(path, delimiter=",", dtype=dtype, ndmin=2)


def _generated(mesh_size: str, test_case: str):
    if test_case == "Test3D":
        return gen.kuhn_tetrahedra(20, 15.24)
    n = int(mesh_size)
    if test_case in ("NitrogenTest", "VGDirichlet"):
        return gen.structured_triangles(n, 1.0)
    if test_case == "SoluteTest":
        raise FileNotFoundError("the SoluteTest meshes are unstructured; pass mesh_dir pointing at data/mesh")
    return gen.structured_triangles(n, 15.24)


def load_and_validate_mesh(mesh_size: str, mesh_dir: Optional[str], test_case: str = "Test1",
                           prefix: Optional[Tuple[str, str]] = None) -> Tuple[np.ndarray, np.ndarray, Dict[str, Any]]:
    is_3d = test_case == "Test3D"
    if mesh_dir is None:
        points, elements = _generated(mesh_size, test_case)
    else:
        base = Path(mesh_dir)
        if test_case == "SoluteTest":
            p_file, t_file = base / "solute" / f"p_Pinns_{mesh_size}.csv", base / "solute" / f"t_Pinns_{mesh_size}.csv"
        elif test_case == "NitrogenTest":
            p_file, t_file = base / "nitrogen" / f"p_{mesh_size}.csv", base / "nitrogen" / f"t_{mesh_size}.csv"
        elif is_3d:
            pp, tp = prefix if prefix else ("p_3D", "t_3D")
            p_file, t_file = base / "richards" / f"{pp}.zip", base / "richards" / f"{tp}.zip"
        else:
            p_file, t_file = base / "richards" / f"p{mesh_size}.csv", base / "richards" / f"t{mesh_size}.csv"
        if not p_file.exists():
            raise FileNotFoundError(f"Points file not found: {p_file}")
        if not t_file.exists():
            raise FileNotFoundError(f"Elements file not found: {t_file}")
        points = _read_csv(p_file, np.float64)
        elements = _read_csv(t_file, np.int64) - 1
    if is_3d:
        if points.ndim != 2 or points.shape[1] != 3:
            raise ValueError("Points array must have 3 columns (x, y, z coordinates) for 3D mesh")
        if elements.ndim != 2 or elements.shape[1] != 4:
            raise ValueError("Elements array must have 4 columns (vertex indices) for tetrahedral mesh")
    else:
        if points.ndim != 2 or points.shape[1] != 2:
            raise ValueError("Points array must have 2 columns (x, y coordinates) for 2D mesh")
        if elements.ndim != 2 or elements.shape[1] != 3:
            raise ValueError("Elements array must have 3 columns (vertex indices) for triangular mesh")
    if np.any(elements < 0) or np.any(elements >= len(points)):
        raise ValueError("Element indices out of bounds")
    info = {"num_points": len(points), "num_elements": len(elements), "dimension": 3 if is_3d else 2,
            "element_type": "tetrahedra" if is_3d else "triangles",
            "x_range": (float(points[:, 0].min()), float(points[:, 0].max())),
            "y_range": (float(points[:, 1].min()), float(points[:, 1].max())),
            "z_range": (float(points[:, 2].min()), float(points[:, 2].max())) if is_3d else None,
            "mesh_type": "solute" if test_case == "SoluteTest" else "richards",
            "mesh_size": mesh_size if test_case != "SoluteTest" else "Pinns"}
    return points, elements, info
