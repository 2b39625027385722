"""C ABI: the library loads, exports every declared entry point, and rejects
bad input with the documented status codes (no GPU needed)."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

from mlfma_b200 import MLFMA, MlfmaError, default_config, inputs
from mlfma_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        names |= set(re.findall(r"^\s*(?:int|const char\*)\s+(mlfma_\w+)\s*\(", text, re.M))
    return names


def test_header_declares_entry_points():
    names = declared_symbols()
    assert {"mlfma_create_dipoles", "mlfma_create_rwg", "mlfma_setup", "mlfma_matvec", "mlfma_gmres",
            "mlfma_destroy", "mlfma_last_error"} <= names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    assert declared_symbols() <= set(_lib.SIGNATURES)


def test_config_default_matches_reference_fields():
    c = default_config()
    assert (c.digits, c.interp_order, c.over_interp, c.root_leng, c.max_node_srcs) == (3, 3, 2.0, 4.0, 64)
    assert c.ref_compat == 1


def test_rejects_bad_input():
    pw = inputs.PlaneWave()
    d = inputs.make_dipoles(10)
    with pytest.raises(MlfmaError) as e:
        MLFMA.dipoles(inputs.Dipoles(pos=d.pos * 10.0, mom=d.mom), pw)  # outside the root box
    assert e.value.code == _lib.MLFMA_ERR_ARG and "root box" in str(e.value)
    with pytest.raises(MlfmaError) as e:
        MLFMA.dipoles(inputs.Dipoles(pos=d.pos, mom=d.mom * 0.0), pw)
    assert e.value.code == _lib.MLFMA_ERR_ARG
    m = inputs.make_icosphere(1, radius=1.0)
    with pytest.raises(MlfmaError) as e:
        MLFMA.rwg(m, pw, quad_prec=7)
    assert e.value.code == _lib.MLFMA_ERR_ARG
    bad = inputs.RWGMesh(m.vertices, m.faces, m.rwgs.copy())
    bad.rwgs[0, 2] = 10_000
    with pytest.raises(MlfmaError) as e:
        MLFMA.rwg(bad, pw)
    assert e.value.code == _lib.MLFMA_ERR_ARG


def test_device_calls_before_setup_are_state_errors():
    op = MLFMA.dipoles(inputs.make_dipoles(50), inputs.PlaneWave())
    with pytest.raises(MlfmaError) as e:
        op.matvec(np.zeros(50))
    assert e.value.code == _lib.MLFMA_ERR_STATE
    with pytest.raises(MlfmaError) as e:
        op.solve()
    assert e.value.code == _lib.MLFMA_ERR_STATE
    with pytest.raises(MlfmaError):
        op.stage_times()
    with pytest.raises(MlfmaError) as e:
        op.dense_rows([0, 1], np.zeros(50))
    assert e.value.code == _lib.MLFMA_ERR_STATE
    x = np.zeros(50, dtype=np.complex128)
    with pytest.raises(MlfmaError) as e:
        op.matvec_mapped(x.ctypes.data, x.ctypes.data)
    assert e.value.code == _lib.MLFMA_ERR_STATE
    with pytest.raises(MlfmaError) as e:
        op.set_schedule(1)
    assert e.value.code == _lib.MLFMA_ERR_STATE
    with pytest.raises(MlfmaError) as e:
        op.solve_multi(np.zeros((2, 50)), flexible=True)
    assert e.value.code == _lib.MLFMA_ERR_STATE
    op.close()


def test_null_arguments():
    L = _lib.lib()
    assert L.mlfma_setup(None) == _lib.MLFMA_ERR_ARG
    assert L.mlfma_config_default(None) == _lib.MLFMA_ERR_ARG
    assert L.mlfma_destroy(None) == _lib.MLFMA_OK
    assert L.mlfma_last_error()  # message set by the failing call
    assert L.mlfma_dense_rows(None, 1, None, None, None) == _lib.MLFMA_ERR_ARG
    assert L.mlfma_check_bounded_wait(0, None) == _lib.MLFMA_ERR_ARG
    assert L.mlfma_batch_create(0, None, None) == _lib.MLFMA_ERR_ARG
    assert L.mlfma_matvec_mapped(None, None, None, 0) == _lib.MLFMA_ERR_ARG
    assert L.mlfma_set_schedule(None, 0) == _lib.MLFMA_ERR_ARG


def test_host_plan_stats_without_gpu():
    op = MLFMA.dipoles(inputs.make_dipoles(3000, seed=2), inputs.PlaneWave(), max_node_srcs=16)
    st = op.stats()
    assert st["max_level"] == 3 and st["num_levels_far"] == 2
    assert st["near_entries"] > 0 and st["pattern_elems"] > 0
    info, perm = op.far_leaves()
    assert sorted(perm.tolist()) == list(range(3000))
    assert info[:, 3].sum() == 3000
    op.close()


def test_tree_export_and_device_tree_without_gpu():
    op = MLFMA.dipoles(inputs.make_dipoles(3000, seed=2), inputs.PlaneWave(), max_node_srcs=16)
    st = op.stats()
    nodes = op.tree_export(0).reshape(-1, 14)
    assert nodes.shape[0] == st["num_nodes"] and nodes[:, 11].sum() == st["num_leaves"]
    assert nodes[0, 1] == -1 and nodes[0, 13] == 3000  # the root holds every source
    assert sorted(op.tree_export(1).tolist()) == list(range(3000))
    for which, key in ((4, "list2"), (5, "list4")):
        a, total, i = op.tree_export(which), 0, 0
        while i < a.size:  # per node: length, then ids
            total += a[i]
            i += a[i] + 1
        assert i == a.size and total == st[key]
    op.close()
    import torch
    if not torch.cuda.is_available():  # the device build needs a GPU: a clean error
        with pytest.raises(MlfmaError, match="cudaSetDevice"):
            MLFMA.dipoles(inputs.make_dipoles(300, seed=2), inputs.PlaneWave(), device_tree=1)
