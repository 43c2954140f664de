"""The ctypes mirror (sjoin) agrees with include/sj.h: struct layouts as the C
compiler lays them out (offsets and sizes printed by a program built against
the header), and every bound function's arity, argument widths and return
type as the header declares them.  Needs gcc, no device."""
import ctypes as C
import os
import re
import subprocess

import sjoin

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(REPO, "include", "sj.h")

STRUCTS = {
    "sj_params": sjoin.Params, "sj_stats": sjoin.Stats, "sj_batch": sjoin.Batch,
    "sj_grid": sjoin.GridCell, "sj_grid_cell_lookup": sjoin.GridCellLookup,
    "sj_neighbor_table_lookup": sjoin.NeighborTableLookup,
}


def _c_layout(tmp_path):
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "sj.h"', "int main(void) {"]
    for cname, py in STRUCTS.items():
        lines.append(f'printf("{cname} . 0 %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'printf("{cname} {fname} %zu %zu\\n", offsetof({cname}, {fname}), '
                         f'sizeof((({cname} *)0)->{fname}));')
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.check_call(["gcc", "-std=c11", "-I", os.path.dirname(HEADER), str(src), "-o", str(exe)])
    out = {}
    for ln in subprocess.check_output([str(exe)], text=True).splitlines():
        s, f, a, b = ln.split()
        out[(s, f)] = (int(a), int(b))
    return out


def test_struct_layouts_match_the_header(tmp_path):
    c = _c_layout(tmp_path)
    for cname, py in STRUCTS.items():
        assert C.sizeof(py) == c[(cname, ".")][1], cname
        for fname, ftype in py._fields_:
            assert (getattr(py, fname).offset, C.sizeof(ftype)) == c[(cname, fname)], (cname, fname)


def _prototypes():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    text = re.sub(r"//[^\n]*", " ", text)
    protos = {}
    for ret, name, args in re.findall(r"([A-Za-z_][\w \*]*?)\s*\b(sj_\w+)\s*\(([^;{]*?)\)\s*;", text):
        if ret.strip().startswith("typedef"):
            continue
        args = " ".join(args.split())
        plist = [] if args in ("", "void") else [a.strip() for a in args.split(",")]
        protos[name] = (" ".join(ret.split()), plist)
    return protos


def _c_kind(decl: str) -> str:
    decl = decl.strip()
    if "*" in decl or decl.split()[0] == "sj_batch_cb":
        return "ptr"
    base = " ".join(w for w in decl.split()[:-1] if w != "const")   # drop the parameter name
    return {"int": "i32", "sj_status": "i32", "uint32_t": "u32", "unsigned int": "u32", "uint64_t": "u64",
            "float": "f32", "double": "f64", "void": "void"}[base]


def _c_ret_kind(ret: str) -> str:
    ret = ret.replace("const ", "").strip()
    if "*" in ret:
        return "ptr"
    return {"sj_status": "i32", "int": "i32", "uint32_t": "u32", "uint64_t": "u64", "void": "void"}[ret]


def _py_kind(t) -> str:
    if t is None:
        return "void"
    if t in (C.c_void_p, C.c_char_p) or (isinstance(t, type) and issubclass(t, (C._Pointer, C._CFuncPtr))):
        return "ptr"
    for kind, cands in (("i32", (C.c_int, C.c_int32)), ("u32", (C.c_uint, C.c_uint32)),
                        ("u64", (C.c_uint64, C.c_ulonglong)), ("f32", (C.c_float,)), ("f64", (C.c_double,))):
        if t in cands:
            return kind
    raise AssertionError(f"unexpected ctypes type {t}")


def test_every_header_function_is_exported_and_bound_as_declared():
    protos = _prototypes()
    assert len(protos) >= 25
    assert set(protos) <= set(sjoin.EXPORTS) | {"sj_params_default"}, set(protos) - set(sjoin.EXPORTS)
    L = sjoin.load()
    bound = 0
    for name, (ret, params) in protos.items():
        fn = getattr(L, name)
        assert _py_kind(fn.restype) == _c_ret_kind(ret), (name, ret, fn.restype)
        if fn.argtypes is None:
            assert not params, f"{name}: declared with arguments but bound without argtypes"
            continue
        kinds = [_c_kind(p) for p in params]
        assert [_py_kind(t) for t in fn.argtypes] == kinds, (name, params)
        bound += 1
    assert bound >= 20
