"""CPU checks of the C-ABI boundary: the library loads, exports every symbol include/diffphd_b200.h declares,
reports errors through dphd_last_error like the reference's CheckError messages, and its host-side
sparse-inverse factor reproduces the oracle's A^-1 (the set-up self-check; no GPU needed)."""
import ctypes as C

import numpy as np
import pytest

from diffphd_b200 import core, scenes


def test_library_exports_every_declared_symbol():
    L = core.load_library()
    syms = core.exported_symbols()
    assert len(syms) >= 25
    for s in syms:
        assert hasattr(L, s), f"missing export {s}"


def test_device_is_recorded_only_once_built():
    sc = scenes.cantilever(cells=(2, 1, 1), steps=1)
    d = core.from_scene(sc)
    assert d.device() == -1  # nothing built yet: no device bound to the handle
    assert core.load_library().dphd_device(None) == -2


def test_bad_element_dim_reports_error():
    L = core.load_library()
    h = C.c_void_p()
    assert L.dphd_create(3, 5, C.byref(h)) != 0
    assert b"element_dim" in L.dphd_last_error()


def test_builder_errors_mirror_reference_messages():
    sc = scenes.cantilever(cells=(2, 1, 1), steps=1)
    d = core.HexDeformable()
    with pytest.raises(RuntimeError, match="Only material 'none'"):
        d.Initialize(sc.verts, sc.elems, 1e3, "neohookean", 1e6, 0.45)
    d.Initialize(sc.verts, sc.elems, 1e3, "none", 1e6, 0.45)
    with pytest.raises(RuntimeError, match="Inconsistent param size"):
        d.AddPdEnergy("corotated", [1.0, 2.0, 3.0], [])
    with pytest.raises(RuntimeError, match="Unsupported PD energy"):
        d.AddPdEnergy("muscle", [1.0], [])
    with pytest.raises(RuntimeError, match="Element index out of bound"):
        d.AddPdEnergy("corotated", [1.0], [7])
    with pytest.raises(RuntimeError, match="Duplicated vertex"):
        d.SetFrictionalBoundary("planar", [0, 0, 1, 0], [1, 1])
    d.AddPdEnergy("corotated", [1e5], [])
    n = d.dofs()
    with pytest.raises(RuntimeError, match="Missing option max_pd_iter"):
        d.PyForward("pd_eigen_alg_phd", np.zeros(n), np.zeros(n), [], np.zeros(n), 0.01,
                    {"abs_tol": 1e-9, "rel_tol": 1e-6, "verbose": 0, "thread_ct": 1}, None, None, None)
    with pytest.raises(RuntimeError, match="Unsupported method"):
        d.PyForward("newton_pcg", np.zeros(n), np.zeros(n), [], np.zeros(n), 0.01, {}, None, None, None)
    with pytest.raises(RuntimeError, match="Inconsistent vector size"):
        d.PyForward("pd_eigen_alg_phd", np.zeros(n - 1), np.zeros(n), [], np.zeros(n), 0.01, {}, None, None, None)


def test_partial_node_dirichlet_rejected():
    sc = scenes.cantilever(cells=(2, 1, 1), steps=1)
    d = core.from_scene(sc)
    d.SetDirichletBoundaryCondition(3 * (sc.n - 1), 0.0)
    with pytest.raises(RuntimeError, match="whole nodes"):
        d.debug_host_sts(np.zeros(sc.dofs), sc.dt)


@pytest.mark.parametrize("builder", [
    lambda: scenes.cantilever(cells=(6, 2, 3), steps=1),
    lambda: scenes.cantilever(steps=1),
    lambda: scenes.nh_tet_block(cells=(8, 4, 4), dx=0.01, steps=1),
])
def test_host_factor_matches_oracle_solve(oracle_lib, builder):
    sc = builder()
    d = core.from_scene(sc)
    o = oracle_lib.OracleDeformable.from_scene(sc)
    b = np.random.default_rng(0).standard_normal(sc.dofs)
    x = d.debug_host_sts(b, sc.dt)
    xr = o.ainv(b, sc.dt)
    xr[sc.dirichlet_dofs] = 0.0
    assert np.abs(x - xr).max() <= 1e-11 * np.abs(xr).max()
    assert d.s_nnz() > sc.n


def test_malformed_and_truncated_mesh_files_are_rejected(tmp_path):
    """The .bin reader (the reference's Mesh::Initialize, cpp/core/src/mesh/mesh.cpp:4-31) rejects a file with the
    wrong header and a file cut short, with an error instead of reading past the data."""
    import shutil
    from pathlib import Path
    gold = Path(__file__).resolve().parent / "golden" / "ref_hex_16x4x4.bin"
    bad = tmp_path / "bad_header.bin"
    data = bytearray(gold.read_bytes())
    data[0:4] = (7).to_bytes(4, "little")  # vertex dimension 7
    bad.write_bytes(bytes(data))
    cut = tmp_path / "truncated.bin"
    cut.write_bytes(gold.read_bytes()[: len(data) // 2])
    ok = tmp_path / "ok.bin"
    shutil.copy(gold, ok)
    for path, msg in ((bad, "Corrupted mesh file"), (cut, "mesh"), (tmp_path / "missing.bin", "Cannot open")):
        d = core.HexDeformable()
        with pytest.raises(RuntimeError, match=msg):
            d.Initialize(str(path), 1e3, "none", 1e6, 0.45)
    d = core.HexDeformable()
    d.Initialize(str(ok), 1e3, "none", 1e6, 0.45)
    assert d.dofs() == 3 * 425
