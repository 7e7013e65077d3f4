"""CPU-side checks: the C-ABI library loads and exports every declared symbol; the tree packer."""

import ctypes
import os
import re

import numpy as np
import pytest
import torch

from betterrobot_b200 import _lib, synthetic as syn
from betterrobot_b200.tree import TreeArrays

from conftest import REPO


def _declared_symbols():
    names = []
    for fn in os.listdir(os.path.join(REPO, "include")):
        if fn.endswith(".h"):
            src = open(os.path.join(REPO, "include", fn)).read()
            names += re.findall(r"^\s*BR_API\s+(?:int|int64_t|const char\s*\*)\s+(br_\w+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = _declared_symbols()
    assert "br_frame_jacobians" in names and "br_forward_kinematics" in names
    # the ctypes table covers every declared symbol and nothing else
    assert sorted(_lib.SIGNATURES) == names


def _prototypes():
    """name -> list of parameter declarations, from every BR_API prototype of the headers."""
    out = {}
    for fn in os.listdir(os.path.join(REPO, "include")):
        if fn.endswith(".h"):
            src = open(os.path.join(REPO, "include", fn)).read()
            for m in re.finditer(r"BR_API\s+[^;{]*?\b(br_\w+)\s*\(([^)]*)\)\s*;", src, flags=re.S):
                params = [" ".join(x.split()) for x in m.group(2).split(",")]
                out[m.group(1)] = [] if params == ["void"] or params == [""] else params
    return out


def test_ctypes_signatures_match_the_prototypes():
    """Every entry point's ctypes argtypes have the prototype's arity, and each parameter's
    kind: a pointer (to a struct: POINTER of the mirror struct) / int32_t / int64_t."""
    protos = _prototypes()
    assert sorted(protos) == sorted(_lib.SIGNATURES)
    for name, params in protos.items():
        args = _lib.SIGNATURES[name][1]
        assert len(args) == len(params), name
        for decl, ct in zip(params, args):
            if "*" in decl:
                assert ct is ctypes.c_void_p or issubclass(ct, ctypes._Pointer), (name, decl, ct)
            elif decl.startswith("int64_t"):
                assert ct is ctypes.c_int64, (name, decl, ct)
            elif decl.startswith("int32_t"):
                assert ct is ctypes.c_int32, (name, decl, ct)
            else:
                raise AssertionError(f"{name}: unexpected parameter type {decl!r}")


def test_library_loads_and_exports_every_declared_symbol():
    lib = _lib.load()
    for name in _declared_symbols():
        assert hasattr(lib, name), name
    assert b"sm_100a" in lib.br_version()


def _header_structs():
    """typedef name -> [(C type, field name)] in declaration order, from the headers."""
    out = {}
    for fn in os.listdir(os.path.join(REPO, "include")):
        if fn.endswith(".h"):
            src = open(os.path.join(REPO, "include", fn)).read()
            src = re.sub(r"/\*.*?\*/", " ", src, flags=re.S)
            for m in re.finditer(r"typedef\s+struct\s+\w+\s*\{(.*?)\}\s*(\w+)\s*;", src, flags=re.S):
                fields = []
                for decl in m.group(1).split(";"):
                    decl = " ".join(decl.split())
                    if not decl:
                        continue
                    first = re.match(r"((?:const\s+)?\w+\s*\**)\s*(.*)", decl)
                    ctype, names = first.group(1).replace(" ", ""), first.group(2)
                    for nm in names.split(","):
                        nm = nm.strip()
                        stars = len(nm) - len(nm.lstrip("*"))
                        fields.append((ctype + "*" * stars, nm.lstrip("*").strip()))
                out[m.group(2)] = fields
    return out


@pytest.mark.parametrize("c_name,mirror", [("br_tree_t", "BrTree"), ("br_ik_settings_t", "IKSettings"),
                                           ("br_ik_batch_t", "IKBatch"), ("br_ik_result_t", "IKResultBuf"),
                                           ("br_traj_settings_t", "TrajSettings")])
def test_struct_mirrors_match_header(c_name, mirror):
    """Field names, order and kinds of each ctypes mirror equal the header's struct."""
    fields = _header_structs()[c_name]
    py = getattr(_lib, mirror)._fields_
    assert [n for _, n in fields] == [n for n, _ in py], c_name
    for (ctype, name), (_, ct) in zip(fields, py):
        if ctype.endswith("*"):
            assert ct is ctypes.c_void_p or issubclass(ct, ctypes._Pointer), (name, ctype, ct)
        else:
            assert ct is {"float": ctypes.c_float, "int32_t": ctypes.c_int32, "int64_t": ctypes.c_int64}[ctype], name


def test_tree_struct_layout_matches_header():
    # 8 int32 (sizes, rounds, kinds, dof_entries, dof_depth), then 14 table pointers and dof_sched
    assert ctypes.sizeof(_lib.BrTree) == 32 + 15 * 8
    assert _lib.BrTree.parent.offset == 32
    assert _lib.BrTree.dof_sched.offset == 32 + 14 * 8


@pytest.mark.parametrize("spec", [syn.chain_spec(), syn.humanoid_spec(), syn.dual_arm_spec()])
def test_tree_arrays(spec):
    m = syn.model_from_spec(spec)
    a = TreeArrays(m)
    assert a.nj == m.njoints and a.nv == m.nv
    for j in range(m.njoints):
        sup = set(m.supports[j])
        bits = {k for k in range(m.njoints) if (int(a.support[j]) >> k) & 1}
        assert bits == sup
    depth = max(len(s) - 1 for s in m.supports)
    assert 2 ** a.rounds >= depth + 1 and 2 ** max(a.rounds - 1, 0) < depth + 1
    for c in range(m.nv):
        j = a.col_joint[c]
        assert m.idx_vs[j] <= c < m.idx_vs[j] + m.nvs[j]
    buf, offs = a.blob()
    assert all(o % 16 == 0 for o in offs.values())


def test_unsupported_joint_kind_rejected():
    from betterrobot_b200.exceptions import UnsupportedJointError
    from betterrobot_b200.model import joint_model
    for kind in ("helical", "mimic", "composite"):  # not buildable by the reference's build_model either
        with pytest.raises(UnsupportedJointError):
            joint_model(kind)


def test_cpu_tensor_rejected_without_fallback():
    """No CPU fallback: a CPU tensor never reaches a kernel and raises."""
    from betterrobot_b200 import forward_kinematics
    from betterrobot_b200.exceptions import BackendNotAvailableError, DeviceMismatchError
    m = syn.model_from_spec(syn.chain_spec())
    with pytest.raises((BackendNotAvailableError, DeviceMismatchError)):
        forward_kinematics(m, torch.zeros(4, m.nq))


def test_shape_error_before_device_check():
    from betterrobot_b200 import forward_kinematics
    from betterrobot_b200.exceptions import ShapeError
    m = syn.model_from_spec(syn.chain_spec())
    with pytest.raises(ShapeError):
        forward_kinematics(m, torch.zeros(4, m.nq + 1))


def test_device_tree_cache_keeps_no_model_alive():
    import gc
    from betterrobot_b200 import tree as tr
    m = syn.model_from_spec(syn.chain_spec())
    dt = tr.device_tree(m, "cpu")
    key = (id(m), "cpu")
    assert tr._CACHE[key] is dt and dt.model is m
    assert tr.device_tree(m, "cpu") is dt  # cached
    del m
    gc.collect()
    assert key not in tr._CACHE and dt.model is None
