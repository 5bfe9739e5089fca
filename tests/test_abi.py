"""The C ABI library without a GPU: it loads, exports every declared symbol, and
rejects bad input before touching the device."""
import ctypes as C
import os
import subprocess

import pytest

import diskgpu as D
from helpers import ROOT, parse_header_symbols


def test_library_exports_every_declared_symbol():
    L = D.lib()
    declared = parse_header_symbols()
    assert len(declared) >= 19
    missing = [s for s in declared if not hasattr(L, s)]
    assert not missing, missing
    assert set(D.EXPORTS) == set(declared)


def test_params_struct_layout_matches_header(tmp_path):
    """Compile a probe against include/diskgpu.h and compare offsets with the ctypes mirror."""
    src = tmp_path / "probe.c"
    fields = [f[0] for f in D.Params._fields_]
    body = "\n".join(f'  printf("%s %%zu\\n", offsetof(dg_params, {f}));' % f for f in fields)
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "diskgpu.h"\nint main(){\n'
                   + body + '\n  printf("size %zu\\n", sizeof(dg_params));\n'
                   + '  printf("rec %zu\\n", sizeof(dg_record));\n  return 0;\n}\n')
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = dict(l.split() for l in subprocess.run([str(exe)], capture_output=True, text=True).stdout.splitlines())
    for f in fields:
        assert int(out[f]) == getattr(D.Params, f).offset, f
    assert int(out["size"]) == C.sizeof(D.Params)
    assert int(out["rec"]) == C.sizeof(D.Record)


def test_defaults_are_the_reference_cli_defaults():
    p = D.default_params()
    # diskmain.cpp:17-29
    assert (p.Nu, p.Nphi, p.eps, p.selfgrav, p.amp) == (128, 128, 0.02, 1, 1e-3)
    assert (p.Rin, p.Rout, p.R0, p.w2, p.S0) == (0.25, 1.0, 0.45, 0.05, 0.372)
    assert (p.Kpoly, p.gamma_gas, p.gmstar, p.G) == (0.25, 2.0, 0.6, 1.0)


@pytest.mark.parametrize("kw,code", [
    (dict(Nu=1), -1), (dict(Nphi=1), -1), (dict(Rin=0.0), -1), (dict(Rout=0.1), -1),
    (dict(Nphi=14), -4), (dict(Nu=7), -4), (dict(precision=7), -1), (dict(eps=-1.0), -1),
    (dict(Nu=8192), -4), (dict(Nphi=16384), -4),  # the largest grid is 4096 x 8192
    (dict(gamma_gas=0.0), -1), (dict(Kpoly=-0.25), -1), (dict(Nphi=14 * 7), -4),
])
def test_invalid_params_rejected_before_device(kw, code):
    with pytest.raises(D.DiskGPUError) as e:
        D.Disk(**{**dict(Nu=32, Nphi=32), **kw})
    assert e.value.code == code


def test_status_strings():
    L = D.lib()
    assert L.dg_status_string(0) == b"ok"
    assert L.dg_status_string(-3) == b"non-finite state or dt"
    L.dg_destroy(None)  # no-op
