"""Generates the committed mesh fixtures in tests/golden/ by running the reference's own pure-Python
mesh writers (python/py_diff_pd/common/hex_mesh.py:generate_hex_mesh and
python/py_diff_pd/common/tet_mesh.py:generate_tet_mesh).

The reference's compiled core is not importable here, so the two modules are imported with stub
entries for `py_diff_pd.core.py_diff_pd_core` and `trimesh`, which the writers never call.
Run from the repository root:  python tests/golden/make_golden.py <reference checkout>
(the directory that holds the reference's python/ tree; the fixtures it writes are committed, so tests do
not need the checkout).
"""
import sys
import types
from pathlib import Path

import numpy as np

OUT = Path(__file__).resolve().parent


def _import_reference(ref_root: Path):
    core = types.ModuleType("py_diff_pd.core.py_diff_pd_core")
    for name in ("HexMesh3d", "TetMesh3d", "StdRealVector", "StdIntVector", "StdMap", "StdRealMatrix",
                 "StdRealArray3d", "StdRealArray2d", "StdRealVector2d"):
        setattr(core, name, object)
    sys.modules["py_diff_pd.core.py_diff_pd_core"] = core
    for mod in ("trimesh", "tetgen", "pyvista"):
        sys.modules.setdefault(mod, types.ModuleType(mod))
    sys.path.insert(0, str(ref_root / "python"))
    from py_diff_pd.common import hex_mesh, tet_mesh  # noqa: E402
    return hex_mesh, tet_mesh


def main(argv):
    if len(argv) != 2 or not (Path(argv[1]) / "python" / "py_diff_pd").is_dir():
        raise SystemExit("usage: python tests/golden/make_golden.py <reference checkout with python/py_diff_pd>")
    hex_mesh, tet_mesh = _import_reference(Path(argv[1]))
    # 1) the cantilever box (16x4x4 cells, dx 0.01)
    hex_mesh.generate_hex_mesh(np.ones((16, 4, 4)), 0.01, [0.0, 0.0, 0.0], str(OUT / "ref_hex_16x4x4.bin"))
    # 2) a sparse voxel shape, to pin node compaction and element corner order
    vox = np.ones((3, 3, 2))
    vox[1, 1, :] = 0
    vox[2, 0, 1] = 0
    hex_mesh.generate_hex_mesh(vox, 0.5, [0.1, -0.2, 0.3], str(OUT / "ref_hex_holes.bin"))
    # 3) the tet writer's layout, on a fixed 2-tet mesh
    verts = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [1, 1, 1]], dtype=np.float64)
    faces = np.array([[0, 1, 2, 3], [1, 2, 3, 4]])
    tet_mesh.generate_tet_mesh(verts, faces, str(OUT / "ref_tet_2.bin"))
    print("wrote", sorted(p.name for p in OUT.glob("ref_*.bin")))


if __name__ == "__main__":
    main(sys.argv)
