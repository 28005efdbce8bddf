"""The C-ABI boundary without a GPU: the library builds, loads, exports every
symbol include/tide_b200.h declares, and its argtypes equal the reference
loader's (src/tide/backend_utils.py:227-308, captured in golden/abi_specs.json)."""

from __future__ import annotations

import json
import re
import subprocess

import pytest
import torch

from conftest import GOLDEN, REPO
from tide_b200 import _native as nat


def header_symbols() -> set[str]:
    names: set[str] = set()
    for h in sorted((REPO / "include").glob("*.h")):
        out = subprocess.run(["gcc", "-E", "-P", "-x", "c", str(h)], capture_output=True,
                             text=True, check=True).stdout
        names |= set(re.findall(r"\b((?:maxwell_tm|maxwell_3d|tide)_\w+)\s*\(", out))
    return names


def test_library_exports_every_declared_symbol():
    lib = nat.load()
    declared = header_symbols()
    assert set(nat.exported_symbols()) <= declared
    assert set(nat.exported_symbols()) == declared
    assert len(declared) >= 36
    for name in declared:
        assert hasattr(lib, name), name


def test_library_metadata_calls_without_gpu():
    lib = nat.load()
    assert lib.tide_cuda_arches() == b"100a"
    lib.tide_b200_clear_error()
    assert lib.tide_b200_last_status() == 0


@pytest.mark.parametrize("template", sorted(nat.SPECS))
@pytest.mark.parametrize("dtype", ["float", "double"])
def test_argtypes_match_reference_loader(template, dtype):
    """Every entry point the library binds with a reference template has the
    reference loader's argtypes (golden/abi_specs.json, captured from
    src/tide/backend_utils.py by golden/make_golden.py)."""
    specs = json.loads((GOLDEN / "abi_specs.json").read_text())
    ref = specs[f"{template}_{dtype}"]
    mine = [a.__name__ for a in nat.argtypes(template, dtype)]
    assert mine == ref


def test_symbol_naming_matches_reference():
    assert nat.symbol_name("maxwell_tm", "backward", 4, "double") == "maxwell_tm_4_double_backward_cuda"


def test_cpu_tensors_fail_loudly():
    """No silent CPU fallback: the product path refuses CPU tensors."""
    with pytest.raises(nat.NativeError):
        nat.get_backend_function("maxwell_tm", "forward", 2, torch.float32, torch.device("cpu"))


def test_serve_job_struct_layout_matches_header(tmp_path):
    """The ctypes mirror of TideServeJob has the C layout (offsets and size
    from a program compiled against include/tide_b200_serve.h)."""
    from tide_b200 import serve as sv

    fields = [f[0] for f in sv._CJob._fields_]
    body = "\n".join(f'  printf("{f} %zu\\n", offsetof(TideServeJob, {f}));' for f in fields)
    src = tmp_path / "layout.c"
    src.write_text(
        "#include <stddef.h>\n#include <stdio.h>\n#include \"tide_b200_serve.h\"\n"
        "int main(void) {\n" + body +
        '\n  printf("size %zu\\n", sizeof(TideServeJob));\n  return 0;\n}\n')
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", str(REPO / "include"), str(src), "-o", str(exe)], check=True)
    out = dict(line.split() for line in subprocess.run([str(exe)], capture_output=True, text=True,
                                                       check=True).stdout.splitlines())
    for f in fields:
        assert int(out[f]) == getattr(sv._CJob, f).offset, f
    assert int(out["size"]) == __import__("ctypes").sizeof(sv._CJob)
