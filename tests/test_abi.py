"""The C ABI library loads on a CPU-only machine, exports every function include/*.h
declares, checks its inputs on the host, and fails loudly (no CPU fallback) without a GPU."""
import ctypes as C
import glob
import os
import re

import numpy as np
import pytest

import dmplex_b200 as d
from dmplex_b200 import _lib
from conftest import ROOT, gpu_available, tables, trisk_grid


def declared_functions():
    names = set()
    for header in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(header).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(trisk_\w+)\s*\(", text))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(_lib.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing


def test_struct_layouts_match():
    for which, cls in enumerate((_lib.TriskGrid, _lib.TriskCoefficients, _lib.TriskConfig, _lib.TriskPlex)):
        assert _lib.lib.trisk_struct_size(which) == C.sizeof(cls)
    from oracle.oracle import OracleModelStruct
    assert C.sizeof(OracleModelStruct) == C.sizeof(_lib.TriskCoefficients)


def test_bad_tables_are_rejected_on_the_host():
    t = dict(tables(3, "trisk", "cell"))
    bad = t["cell_edges"].copy()
    bad[4, 2] = t["ne"] + 7
    t["cell_edges"] = bad
    with pytest.raises(d.TriskError) as e:
        d.TRiSKShallowWater.from_coefficients(t, pv_flux="trisk", kinetic_energy="cell")
    assert e.value.status == 2 and "cell_edges" in str(e.value)
    t = dict(tables(3, "gassmann", "cell"))
    t["g_edges"] = None
    with pytest.raises(d.TriskError) as e:
        d.TRiSKShallowWater.from_coefficients(t, pv_flux="gassmann", kinetic_energy="cell")
    assert e.value.status == 1


def test_bad_arguments():
    with pytest.raises(ValueError):
        d.TRiSKShallowWater(trisk_grid(2), pv_flux="upwind")
    with pytest.raises(ValueError):
        d.TRiSKShallowWater(trisk_grid(2), kinetic_energy="edge")
    with pytest.raises(d.TriskError) as e:
        d.create_hexagon_mesh(-1)
    assert e.value.status == 1


def test_no_gpu_fails_loudly():
    if gpu_available():
        pytest.skip("a GPU is present")
    with pytest.raises(d.TriskError) as e:
        d.TRiSKShallowWater(trisk_grid(2))
    assert e.value.status == 3


def test_last_error_is_thread_local_and_bounded():
    with pytest.raises(d.TriskError):
        d.create_hexagon_mesh(11)
    buf = C.create_string_buffer(8)
    n = _lib.lib.trisk_last_error(buf, len(buf))
    assert n > 7 and len(buf.value) == 7


def test_tables_are_deterministic():
    """The host table builder gives identical arrays on every call (the parity fixtures
    depend on it)."""
    a = d.model_tables(d.TRiSKGrid(d.create_hexagon_mesh(4, centroidal=True)), pv_flux="gassmann",
                       kinetic_energy="mixed")
    b = d.model_tables(d.TRiSKGrid(d.create_hexagon_mesh(4, centroidal=True)), pv_flux="gassmann",
                       kinetic_energy="mixed")
    for k, v in a.items():
        if isinstance(v, np.ndarray):
            assert np.array_equal(v, b[k]), k
