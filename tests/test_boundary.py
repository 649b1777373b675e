"""The C-ABI boundary and the host logic, without a GPU."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_every_declared_symbol():
    from gnu_femlisp_b200 import _capi
    lib = _capi.load()
    declared = _capi.header_symbols()
    assert len(declared) >= 30
    missing = [s for s in declared if not hasattr(lib, s)]
    assert not missing, missing
    # every declared symbol has a ctypes signature in the binding
    assert set(declared) <= set(_capi.SIGNATURES), set(declared) - set(_capi.SIGNATURES)


def test_header_cites_reference_for_each_entry_point():
    text = open(os.path.join(ROOT, "include", "fmgpu.h")).read()
    # each prototype is preceded by a comment; most cite a Femlisp file:line
    assert len(re.findall(r"\.lisp:\d+", text)) >= 25


def test_init_fails_loudly_without_gpu():
    import torch
    from gnu_femlisp_b200 import Context, FmgError
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(FmgError):
        Context(0)


@pytest.mark.parametrize("cname,pyname", [("fmg_solve_cfg", "SolveCfg"), ("fmg_mixed_cfg", "MixedCfg")])
def test_cfg_layout_matches_header(tmp_path, cname, pyname):
    """The ctypes mirrors of the configuration structs have the C compiler's layout."""
    import shutil
    import subprocess
    from gnu_femlisp_b200 import _capi
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    cls = getattr(_capi, pyname)
    src = tmp_path / "layout.c"
    fields = [f for f, _ in cls._fields_]
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "fmgpu.h"\nint main(void){'
                   f'printf("%zu", sizeof({cname}));'
                   + "".join(f'printf(" %zu", offsetof({cname}, {f}));' for f in fields)
                   + "return 0;}\n")
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True).stdout.split()]
    assert out[0] == ctypes.sizeof(cls)
    assert out[1:] == [getattr(cls, f).offset for f in fields]


def test_ctypes_signatures_match_header():
    """Every declared function has a ctypes signature with the header's
    number of arguments."""
    from gnu_femlisp_b200 import _capi
    h = open(os.path.join(ROOT, "include", "fmgpu.h")).read()
    h = re.sub(r"/\*.*?\*/", "", h, flags=re.S)
    arity = {}
    for m in re.finditer(r"\b(?:int|long|void)\s+(fmg_\w+)\s*\(([^)]*)\)\s*;", h):
        args = [a for a in m.group(2).split(",") if a.strip() and a.strip() != "void"]
        arity[m.group(1)] = len(args)
    assert set(arity) == set(_capi.SIGNATURES), set(arity) ^ set(_capi.SIGNATURES)
    bad = {n: (len(_capi.SIGNATURES[n][1]), k) for n, k in arity.items() if len(_capi.SIGNATURES[n][1]) != k}
    assert not bad, bad


def test_femlisp_forms():
    from gnu_femlisp_b200.iteration import _conditions
    assert _conditions("(or (< :defnorm 1.0e-12) (> :step 10))") == {"atol": 1e-12, "maxsteps": 10}
    assert _conditions("(< :reduction 1.0e-10)") == {"rtol": 1e-10}
    with pytest.raises(ValueError):
        _conditions("(> :time 3)")


def test_make_cfg_maps_iteration_objects():
    import gnu_femlisp_b200 as G
    from gnu_femlisp_b200 import _capi
    from gnu_femlisp_b200.iteration import make_cfg
    cs = G.geometric_cs(smoother=G.SOR(omega=1.2), pre_steps=2, post_steps=2, base_level=2)
    cfg, base, step_success = make_cfg(G.CG(preconditioner=cs), "(< :reduction 1e-10)", "(> :step 50)")
    assert cfg.method == _capi.FMG_METHOD_CG_MG and cfg.smoother == _capi.FMG_SOR
    assert cfg.damp == 1.2 and cfg.pre_steps == 2 and base == 2 and cfg.maxsteps == 50
    assert not step_success and cfg.rtol == 1e-10


def test_gauss_sampling_layout():
    from gnu_femlisp_b200.iteration import gauss_points_1d, sample_at_gauss_points
    v = sample_at_gauss_points(lambda x: x[..., 0] + 10 * x[..., 1], 2, 1, 2).reshape(4, 4)
    xi = gauss_points_1d(1)
    # cell 1 = (cx=1, cy=0), point 2 = (qx=0, qy=1)
    assert v[1, 2] == pytest.approx((1 + xi[0]) * 0.5 + 10 * (0 + xi[1]) * 0.5)


def test_algebraic_system_checks_and_default_smoother():
    # no GPU needed: the shapes are checked on construction, the device grid
    # is made only when a solve asks for it
    import numpy as np
    import scipy.sparse as sp
    import gnu_femlisp_b200 as G
    from gnu_femlisp_b200.iteration import make_cfg, CG, geometric_cs
    A1 = sp.diags([2.0] * 4).tocsr()
    A0 = sp.diags([2.0] * 2).tocsr()
    P = sp.csr_matrix(np.array([[1.0, 0.0], [1.0, 0.0], [0.0, 1.0], [0.0, 1.0]]))
    s = G.AlgebraicSystem([A0, A1], [P], np.ones(4))
    assert s.sizes == [2, 4] and s.fe is None
    with pytest.raises(ValueError):
        G.AlgebraicSystem([A0, A1], [], np.ones(4))
    with pytest.raises(ValueError):
        G.AlgebraicSystem([A0, A1], [P.T.tocsr()], np.ones(4))
    with pytest.raises(ValueError):
        G.AlgebraicSystem([A0, A1], [P], np.ones(3))
    cfg, _, _ = make_cfg(CG(preconditioner=geometric_cs()), "(< :reduction 1e-10)", "(> :step 50)", order=None)
    assert cfg.smoother == G._capi.FMG_JACOBI
