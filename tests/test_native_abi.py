"""The C-ABI library: loads without a GPU, exports every entry point that
include/fugal_b200.h declares, and rejects bad arguments before any launch."""

import ctypes
import re
from pathlib import Path

import pytest

from cugal_b200 import _native as N

HEADER = Path(__file__).resolve().parents[1] / "include" / "fugal_b200.h"


def declared_functions() -> list[str]:
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fugal_[a-z0-9_]+)\s*\(", text)))


def test_library_loads_and_exports_every_declared_symbol():
    lib = N.lib()
    names = declared_functions()
    assert len(names) >= 20
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) == set(N.SIGNATURES), set(names) ^ set(N.SIGNATURES)


def test_version_and_status_strings():
    lib = N.lib()
    assert lib.fugal_version() >= 1
    assert lib.fugal_status_string(0) == b"ok"
    assert lib.fugal_status_string(6) == b"device wait timed out"


def test_record_layout_matches_header():
    # int32 x4, double x2, double[256]
    assert N.RECORD_BYTES == 16 + 16 + 8 * N.MAX_RECORDED_ERRORS


def test_workspace_queries_are_host_only():
    assert N.workspace_size("fugal_gradient_workspace_size", 1000) == 1000 * 1000 * 4
    assert N.workspace_size("fugal_sinkhorn_workspace_size", 32768, N.FUGAL_BF16) > 0
    assert N.workspace_size("fugal_greedy_lap_workspace_size", 4096, 8) >= 4096 * 8 * 8
    assert N.workspace_size("fugal_create_adjacency_workspace_size", 10, 5) > 0


@pytest.mark.parametrize("call", [
    lambda: N.call("fugal_fw_update", 16, None, 16, None, 16, None, None, None, None, 0.5, 1.0, None, 0, None),
    lambda: N.call("fugal_graph_features", None, None, 10, None, None, None, None, None),
    lambda: N.call("fugal_greedy_lap", None, 16, 16, 1, None, 8, 1, None, None, 0, None),
    lambda: N.call("fugal_sinkhorn_solve", None, None, 0, None),
])
def test_bad_arguments_raise_before_launch(call):
    with pytest.raises(N.NativeError):
        call()


def test_bad_sizes_raise():
    with pytest.raises(N.NativeError, match="bad shape|bad argument"):
        N.workspace_size("fugal_sinkhorn_workspace_size", 0, N.FUGAL_F32)
    with pytest.raises(N.NativeError):
        N.workspace_size("fugal_greedy_lap_workspace_size", 100, 3 * 0 + 32)
    with pytest.raises(N.NativeError, match="exceeds"):
        N.workspace_size("fugal_sinkhorn_workspace_size", 10**7, N.FUGAL_F32)


def _c_layout(struct: str, fields: list[str]) -> list[int]:
    """sizeof and offsetof of a header struct, as the C compiler lays it out."""
    import shutil
    import subprocess
    import tempfile
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    src = "#include <stdio.h>\n#include <stddef.h>\n#include \"fugal_b200.h\"\nint main(void){"
    src += f'printf("%zu\\n", sizeof({struct}));'
    for f in fields:
        src += f'printf("%zu\\n", offsetof({struct}, {f}));'
    src += "return 0;}"
    with tempfile.TemporaryDirectory() as d:
        c = Path(d) / "t.c"
        c.write_text(src)
        exe = Path(d) / "t"
        subprocess.run([cc, "-I", str(HEADER.parent), str(c), "-o", str(exe)], check=True)
        out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()
    return [int(x) for x in out]


@pytest.mark.parametrize("cls,struct", [(N.SolveParams, "fugal_solve_params"),
                                        (N.SolveRecord, "fugal_solve_record")])
def test_ctypes_structs_match_c_layout(cls, struct):
    names = [f[0] for f in cls._fields_]
    layout = _c_layout(struct, names)
    assert layout[0] == ctypes.sizeof(cls)
    for name, off in zip(names, layout[1:]):
        assert getattr(cls, name).offset == off, name


def declared_arities() -> dict[str, int]:
    """Parameter count of every function the header declares."""
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    out = {}
    for m in re.finditer(r"\b(fugal_[a-z0-9_]+)\s*\(([^;{]*?)\)\s*;", text):
        params = m.group(2).strip()
        out[m.group(1)] = 0 if params in ("", "void") else params.count(",") + 1
    return out


def test_ctypes_signatures_have_the_header_arities():
    arities = declared_arities()
    assert set(arities) == set(N.SIGNATURES), set(arities) ^ set(N.SIGNATURES)
    wrong = {name: (arities[name], len(args)) for name, (_, args) in N.SIGNATURES.items()
             if arities[name] != len(args)}
    assert not wrong, wrong


def test_plan_entry_layout_matches_header():
    # the plan slots are read on the host as int32 pairs (column, float bits)
    assert _c_layout("fugal_plan_entry", ["column", "value"]) == [8, 0, 4]


@pytest.mark.parametrize("call", [
    lambda: N.call("fugal_csr_edge_rows", None, 10, 5, None, None),
    lambda: N.call("fugal_structural_refresh", 16, None, None, None, None, None, 16, None, 16, 30, None, 0, None,
                   None),
    lambda: N.call("fugal_structural_scatter", 16, None, None, 5, None, None, None, None, 32, 1.0, None, 16, None,
                   None),
    lambda: N.call("fugal_structural_scatter", 0, None, None, 5, None, None, None, None, 32, 1.0, None, 16, None,
                   None),
    lambda: N.call("fugal_fw_gradient_structural", 16, None, 16, 1.0, 0, None, 16, None, None, None, 0, 0.0, 1.0,
                   -1.0, None, None, None, 16, None, 16, None),
    lambda: N.call("fugal_fw_update_collect", 16, None, 16, None, 16, None, None, None, None, 0.5, 1.0, None, 0,
                   None, None, 32, None),
])
def test_kept_term_entry_points_reject_bad_arguments_before_launch(call):
    with pytest.raises(N.NativeError):
        call()
