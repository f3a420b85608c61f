"""CPU-only checks of the C ABI library: it loads without a GPU and exports
every entry point that include/cup2d.h declares."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "cup2d.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\**\s+\**(cup2d_\w+)\s*\(", src, flags=re.M)))


def test_library_exports_every_declared_symbol():
    from cubismup_2d_b200 import abi
    abi.lib()
    out = subprocess.run(["nm", "-D", "--defined-only", abi.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (cup2d_\w+)", out))
    declared = declared_functions()
    assert declared, "no declarations parsed"
    missing = [f for f in declared if f not in exported]
    assert not missing, missing
    assert set(abi.EXPORTS) <= exported


def test_context_creation_fails_loudly_without_gpu():
    from cubismup_2d_b200 import Simulation, Cup2DError
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    sim = Simulation("-bpdx 2 -bpdy 1 -poissonType freespace -shapes 'disk radius=0.1'")
    with pytest.raises(Cup2DError):
        sim.init()


def test_argument_parsing_follows_parse_runtime():
    from cubismup_2d_b200 import parse_args
    cfg, shapes = parse_args("-bpdx 16 -bpdy 8 -nu 1.5e-4 -poissonType freespace "
                             "-shapes 'disk radius=0.0375 xpos=0.2 ypos=0.25 bForced=1 bFixed=1 xvel=0.2,"
                             "stefanfish L=0.2 T=1'")
    assert (cfg.bpdx, cfg.bpdy) == (16, 8)
    assert cfg.CFL == 0.1 and cfg.lambda_ == 1e3 / 0.1 and cfg.extent == 1   # Simulation.cpp:92-93
    assert cfg.fadeLen == 0.01 and cfg.poisson == 0
    assert [k for k, _ in shapes] == [0, 1]
    d = shapes[0][1]
    assert d.radius == 0.0375 and d.xvel == 0.2 and d.bForced == 1 and d.bFixed == 1
    f = shapes[1][1]
    assert f.L == 0.2 and f.T == 1


def test_missing_grid_arguments_are_an_error():
    from cubismup_2d_b200 import parse_args, Cup2DError
    with pytest.raises(Cup2DError):
        parse_args("-nu 1e-3")


def test_ensemble_entry_points_reject_bad_arguments():
    """No GPU needed: the ensemble calls check their arguments before any
    CUDA call."""
    import ctypes
    from cubismup_2d_b200 import abi
    L = abi.lib()
    out = ctypes.c_void_p()
    assert L.cup2d_ensemble_create(None, 0, ctypes.byref(out)) == abi.EINVAL
    assert L.cup2d_ensemble_create(None, 2, ctypes.byref(out)) == abi.EINVAL
    assert L.cup2d_ensemble_advance(None, 1) == abi.EINVAL
    assert L.cup2d_ensemble_advance_timed(None, 1, None) == abi.EINVAL
    assert L.cup2d_ensemble_sync(None) == abi.EINVAL
    cnt = ctypes.c_int()
    assert L.cup2d_ensemble_get_shapes(None, None, 0, ctypes.byref(cnt)) == abi.EINVAL
    assert L.cup2d_ensemble_destroy(None) == abi.EINVAL
    assert L.cup2d_ensemble_last_error(None) == b"null ensemble"


def test_checkpoint_entry_points_reject_bad_arguments():
    """No GPU needed: the checkpoint calls check their arguments first."""
    import ctypes
    from cubismup_2d_b200 import abi
    L = abi.lib()
    n = ctypes.c_size_t()
    assert L.cup2d_checkpoint_size(None, ctypes.byref(n)) == abi.EINVAL
    assert L.cup2d_checkpoint_save(None, None, 0) == abi.EINVAL
    assert L.cup2d_checkpoint_load(None, None, 0) == abi.EINVAL


def test_header_compiles_as_c_and_matches_the_binding(tmp_path):
    """include/cup2d.h is plain C (a C caller, not only nvcc, can include it),
    and the ctypes structures of the Python binding have its layouts."""
    import ctypes
    import shutil
    from cubismup_2d_b200 import abi
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    src = tmp_path / "layout.c"
    src.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "cup2d.h"\n'
        "int main(void) {\n"
        '  printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\\n", sizeof(cup2d_config),\n'
        "         sizeof(cup2d_shape_params), sizeof(cup2d_shape_state), offsetof(cup2d_config, iterative),\n"
        "         offsetof(cup2d_shape_state, forcex), offsetof(cup2d_config, gravity),\n"
        "         offsetof(cup2d_config, autotune), sizeof(cup2d_tuning), offsetof(cup2d_tuning, us),\n"
        "         sizeof(cup2d_adjoint_objective), offsetof(cup2d_adjoint_objective, gait_step));\n"
        "  return 0;\n}\n")
    exe = tmp_path / "layout"
    r = subprocess.run([cc, "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                        str(src), "-o", str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True).stdout.split()]
    assert got == [ctypes.sizeof(abi.Config), ctypes.sizeof(abi.ShapeParams), ctypes.sizeof(abi.ShapeState),
                   abi.Config.iterative.offset, abi.ShapeState.forcex.offset, abi.Config.gravity.offset,
                   abi.Config.autotune.offset, ctypes.sizeof(abi.Tuning), abi.Tuning.us.offset,
                   ctypes.sizeof(abi.AdjointObjective), abi.AdjointObjective.gait_step.offset]
