"""Host-side set-up and the C-ABI library, on the CPU (no kernel launches)."""

import ctypes
import os
import re

import numpy as np
import pytest
import scipy.sparse as sp

from pycfd_b200 import hierarchy, _lib
from pycfd_b200.config import BCKind, BCSpec, SimulationConfig
from pycfd_b200.mesh import StructuredMesh
from pycfd_b200.obstacles import circle_mask
from oracle.multigrid import Hierarchy, solve_coarsest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def csr(g, prefix):
    return sp.csr_matrix((g[prefix + "_data"], g[prefix + "_indices"], g[prefix + "_indptr"]),
                         shape=tuple(g[prefix + "_shape"]))


@pytest.mark.parametrize("name", ["walls", "periodic", "periodic_x", "obstacle", "dirichlet",
                                  "isolated"])
def test_product_assembly_matches_reference(golden, name):
    g = golden("poisson.npz")
    nx, ny, lx, ly, px, py = g[name + "_geom"]
    nx, ny = int(nx), int(ny)
    solid = g[name + "_solid"]
    op = hierarchy.assemble(nx, ny, lx / nx, ly / ny, bool(px), bool(py),
                            solid if solid.any() else None,
                            {"right": 0.3} if name == "dirichlet" else None)
    A = op.A.tocsr()
    A.sort_indices()
    ref = csr(g, name + "_A")
    assert np.array_equal(A.indptr, ref.indptr) and np.array_equal(A.indices, ref.indices)
    assert np.array_equal(A.data, ref.data)
    assert np.array_equal(op.fluid, g[name + "_fluid"])
    assert op.pin == int(g[name + "_pin"]) and op.singular == bool(g[name + "_singular"])
    assert np.array_equal(op.bc_rhs, g[name + "_bc"])


@pytest.mark.parametrize("name", ["walls", "periodic", "obstacle", "odd_dirichlet"])
def test_product_hierarchy_matches_reference(golden, name):
    g = golden("multigrid.npz")
    A0 = csr(g, name + "_A0")
    shape = tuple(int(s) for s in g[name + "_shape0"])
    op = hierarchy.FineOperator(A0, shape, g[name + "_active0"], name != "odd_dirichlet", 0,
                                np.zeros(A0.shape[0]))
    levels, cinv = hierarchy.build_hierarchy(op)
    assert len(levels) == int(g[name + "_nlev"])
    for l, lv in enumerate(levels):
        assert lv.shape == tuple(g[f"{name}_shape{l}"])
        assert np.array_equal(lv.active, g[f"{name}_active{l}"])
        assert lv.weight == pytest.approx(float(g[f"{name}_w{l}"]), rel=1e-13)
        ref = csr(g, f"{name}_A{l}").toarray()
        assert np.abs(lv.A.toarray() - ref).max() <= 1e-12 * np.abs(ref).max()
        if l:
            assert np.abs(lv.P.toarray() - csr(g, f"{name}_P{l}").toarray()).max() <= 1e-13
    # the dense coarsest map equals the reference's pinned-LU pseudo-inverse
    h = Hierarchy(A0, shape, g[name + "_active0"], name != "odd_dirichlet")
    last = h.levels[-1]
    b = np.random.default_rng(1).standard_normal(last.n)
    assert np.allclose(cinv @ b, solve_coarsest(last, b), rtol=1e-10, atol=1e-12 * np.abs(b).max())


def test_circle_mask_matches_reference(golden):
    g = golden("masks.npz")
    m = circle_mask(StructuredMesh(2048, 1024, 2.0, 1.0), (0.5, 0.5), 0.05).mask
    assert np.array_equal(np.packbits(m.ravel()), g["big_bits"])


def _header_functions():
    text = open(os.path.join(ROOT, "include", "pycfd_b200.h")).read()
    return sorted(set(re.findall(r"^\w[\w\s\*]*?\b(pycfd_\w+)\s*\(", text, flags=re.M)))


def test_library_exports_every_header_symbol():
    path = _lib.LIB_PATH
    if not os.path.exists(path):
        from pycfd_b200 import build
        build.build()
    lib = ctypes.CDLL(path)
    declared = _header_functions()
    assert declared, "no functions parsed from the header"
    assert sorted(_lib.EXPORTS) == declared
    for name in declared:
        assert hasattr(lib, name), name
    L = _lib.load()
    assert L.pycfd_version() == 1


# ctypes mirrors of the header's structs (pycfd_b200/_lib.py) and the C names they bind
_STRUCTS = {"Shape": "pycfd_shape", "AdjArgs": "pycfd_adj_args", "MgLevel": "pycfd_mg_level",
            "SolverDesc": "pycfd_solver_desc", "DtControl": "pycfd_dt_control",
            "BatchOpts": "pycfd_batch_opts", "Stats": "pycfd_stats", "FieldStats": "pycfd_field_stats"}


def test_ctypes_structs_match_the_header_layout(tmp_path):
    """Every struct the Python binding passes through the C ABI has the header's size and
    field offsets: a C program compiled against include/pycfd_b200.h prints sizeof and
    offsetof for each field the ctypes mirror names, in the mirror's order."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "pycfd_b200.h"', "int main(void) {"]
    expect = []
    for py, cname in _STRUCTS.items():
        cls = getattr(_lib, py)
        lines.append(f'  printf("%zu\\n", sizeof({cname}));')
        expect.append((py, "sizeof", ctypes.sizeof(cls)))
        for fname, _ in cls._fields_:
            lines.append(f'  printf("%zu\\n", offsetof({cname}, {fname}));')
            expect.append((py, fname, getattr(cls, fname).offset))
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run([cc, "-std=c99", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                   check=True, capture_output=True)
    got = [int(x) for x in subprocess.run([str(exe)], check=True, capture_output=True,
                                           text=True).stdout.split()]
    assert len(got) == len(expect)
    for (py, what, want), have in zip(expect, got):
        assert have == want, (py, what, have, want)


def test_config_validation_and_roundtrip():
    with pytest.raises(ValueError, match="at least 4x4"):
        SimulationConfig(nx=2, ny=8)
    with pytest.raises(ValueError, match="periodicity"):
        SimulationConfig(boundary_config={"left": BCSpec(BCKind.PERIODIC), "right": BCSpec(),
                                          "bottom": BCSpec(), "top": BCSpec()})
    cfg = SimulationConfig(nx=16, ny=12, re=250.0, pressure_solver="mgcg",
                           boundary_config={"left": BCSpec("inlet", velocity=1.0),
                                            "right": BCSpec("outlet"), "bottom": BCSpec(),
                                            "top": BCSpec("symmetry")})
    back = SimulationConfig.from_json(cfg.to_json()) if hasattr(SimulationConfig, "from_json") \
        else SimulationConfig.from_dict(__import__("json").loads(cfg.to_json()))
    assert back.to_dict() == cfg.to_dict()
    assert cfg.nu == pytest.approx(1.0 / 250.0)
