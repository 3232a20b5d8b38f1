"""The C-ABI library loads (no GPU needed) and exports every entry point that
include/*.h declares, with the signatures the Python mirror binds."""
import ctypes as C
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        txt = open(h).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        for m in re.finditer(r"^\s*[A-Za-z_][\w \*]*?\b(pff_\w+)\s*\(", txt, flags=re.M):
            names.add(m.group(1))
    return names


def test_header_declares_entry_points():
    names = declared_symbols()
    for n in ("pff_compute_receivers", "pff_accumulate", "pff_reroute_flow", "pff_fill_z_add_delta",
              "pff_diffuse_q", "pff_graphflood_core", "pff_last_error_string"):
        assert n in names


def test_library_exports_every_declared_symbol():
    from pyfastflow_b200 import _lib

    lib = _lib.load()
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing
    # the Python binding table covers exactly the declared API
    assert set(_lib.SIGNATURES) == declared_symbols()


def test_host_side_queries_without_gpu():
    from pyfastflow_b200 import _lib

    lib = _lib.load()
    assert lib.pff_version() >= 100
    n = 4096 * 4096
    assert lib.pff_accumulate_workspace_bytes(n) >= 13 * 4 * n
    assert lib.pff_reroute_workspace_bytes(n) > n
    assert lib.pff_fill_workspace_bytes(n) >= 4 * n


def test_argument_errors_are_reported_not_fatal():
    """Bad arguments come back as a status + message, before any device work."""
    from pyfastflow_b200 import _lib

    lib = _lib.load()
    rc = lib.pff_compute_receivers(None, None, None, 1, 1, 1.0, 0, None, None)
    assert rc == 1
    assert b"grid" in lib.pff_last_error_string()
    rc = lib.pff_compute_receivers(None, None, None, 8, 8, 1.0, 7, None, None)
    assert rc == 1 and b"bound_mode" in lib.pff_last_error_string()
    with pytest.raises(_lib.PFFError):
        _lib.call("pff_accumulate", None, None, None, 0, None, 0, None)


def test_python_mirror_rejects_host_tensors():
    import torch

    from pyfastflow_b200 import constants as cte
    from pyfastflow_b200 import flow

    cte.NX, cte.NY, cte.BOUND_MODE = 4, 4, 0
    z = torch.zeros(16)
    with pytest.raises(TypeError):
        flow.compute_receivers(z, torch.zeros(16, dtype=torch.int32), torch.zeros(16))
