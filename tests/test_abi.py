"""The C-ABI library loads, exports exactly what include/fvb.h declares, and
rejects bad configurations with a status (no GPU needed)."""
from __future__ import annotations

import ctypes as C
import re
import subprocess
from pathlib import Path

import pytest

import fvstuff_b200 as F
from fvstuff_b200 import _lib as L

ROOT = Path(__file__).resolve().parent.parent


def _declared():
    text = (ROOT / "include" / "fvb.h").read_text()
    return sorted(set(re.findall(r"FVB_API[^;(]*?\b(fvb_\w+)\s*\(", text)))


def test_header_matches_bindings():
    assert _declared() == sorted(L.declared_symbols())


def test_library_exports_every_declared_symbol():
    out = subprocess.run(["nm", "-D", "--defined-only", str(L.LIB_PATH)], capture_output=True, text=True,
                         check=True).stdout
    exported = sorted(set(re.findall(r" T (fvb_\w+)", out)))
    assert exported == _declared()
    lib = F.lib()
    for name in _declared():
        assert getattr(lib, name) is not None


STRUCTS = {"fvb_config": L.Config, "fvb_case": L.Case, "fvb_stats": L.Stats, "fvb_batch_config": L.BatchConfig,
           "fvb_instance_desc": L.InstanceDesc, "fvb_request": L.Request, "fvb_request_result": L.RequestResult,
           "fvb_serve_config": L.ServeConfig}


def test_struct_layouts_match_bindings(tmp_path):
    """Every struct of the header has the size and field offsets the ctypes
    mirror gives it (compiled here with the system C compiler)."""
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "fvb.h"', "int main(void) {"]
    for cname, cls in STRUCTS.items():
        lines.append('printf("%s %%zu\\n", sizeof(%s));' % (cname, cname))
        for f in cls._fields_:
            lines.append('printf("%s.%s %%zu\\n", offsetof(%s, %s));' % (cname, f[0], cname, f[0]))
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", str(ROOT / "include"), "-o", str(exe), str(src)], check=True)
    got = dict(line.split() for line in subprocess.run([str(exe)], capture_output=True, text=True,
                                                        check=True).stdout.splitlines())
    for cname, cls in STRUCTS.items():
        assert int(got[cname]) == C.sizeof(cls), cname
        for f in cls._fields_:
            assert int(got[cname + "." + f[0]]) == getattr(cls, f[0]).offset, (cname, f[0])


def test_version_and_defaults():
    assert F.lib().fvb_version().startswith(b"fvb")
    cfg = L.Config()
    F.lib().fvb_config_default(C.byref(cfg), 400)
    assert (cfg.n, cfg.order, cfg.cfl, cfg.gamma, cfg.length) == (400, 7, 0.4, 1.4, 1.0)
    c = F.case_params("vortex", -5, -5, 10)
    assert list(c.param[:5]) == [5.0, 1.0, 1.0, 0.0, 0.0]


@pytest.mark.parametrize("kw", [dict(order=4), dict(n=2), dict(precision="f32", order=5), dict(cfl=-1.0),
                                dict(tile=99)])
def test_invalid_configs_rejected(kw):
    args = dict(n=32)
    args.update(kw)
    with pytest.raises(F.FvbError) as e:
        F.Solver(**args)
    assert e.value.status == L.ERR_INVALID


@pytest.mark.parametrize("policy,max_cells", [(7, 0.0), (0, -1.0), (1, float("nan"))])
def test_serve_config_validated(policy, max_cells):
    cfg = L.ServeConfig()
    cfg.policy, cfg.max_cells = policy, max_cells
    assert F.lib().fvb_serve_run(C.byref(cfg), None, 0, None, None) == L.ERR_INVALID


def test_kernel_contract_validates_geometry():
    st = F.lib().fvb_up_rhs(1, 1, 1, 16, 20, 7, 0.1, 1.4, 1, None)  # np < n + 2g
    assert st == L.ERR_INVALID
    st = F.lib().fvb_apply_bc(1, 16, 23, 0, 0, 0, 1, None)  # odd ghost ring
    assert st == L.ERR_INVALID
