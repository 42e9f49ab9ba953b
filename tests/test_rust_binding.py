"""The Rust binding (rust/gargantua-gpu-sys) against the C header it mirrors.

There is no Rust toolchain in this environment, so the crate is checked as
text: every struct of include/gargantua_gpu.h has a #[repr(C)] Rust struct
with the same fields, types and order, whose layout (rebuilt with ctypes from
the Rust field types) has the size the library reports; every GG_API entry
point is declared with the same number of parameters; every constant has
the header's value.  rust/gargantua-gpu keeps the signatures of
raytracer::curved::render / render_with_disk (renderer.rs:82-101)."""
from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
HEADER = (ROOT / "include" / "gargantua_gpu.h").read_text()
SYS = (ROOT / "rust" / "gargantua-gpu-sys" / "src" / "lib.rs").read_text()
SAFE = (ROOT / "rust" / "gargantua-gpu" / "src" / "lib.rs").read_text()

C2RUST = {"int32_t": "i32", "uint32_t": "u32", "uint64_t": "u64", "double": "f64",
          "float": "f32", "int": "c_int"}
RUST2CT = {"i32": C.c_int32, "u32": C.c_uint32, "u64": C.c_uint64, "f64": C.c_double,
           "f32": C.c_float}


def strip_comments(s: str) -> str:
    s = re.sub(r"/\*.*?\*/", "", s, flags=re.S)
    return re.sub(r"//[^\n]*", "", s)


def c_structs() -> dict:
    out = {}
    for m in re.finditer(r"typedef struct (\w+) \{(.*?)\} \1;", strip_comments(HEADER), re.S):
        fields = []
        for decl in m.group(2).split(";"):
            decl = decl.strip()
            if not decl:
                continue
            t, name = re.match(r"(.+?)\s*(\**\w+(?:\[\w+\])?)$", decl).groups()
            ptr = name.count("*") + t.count("*")
            name = name.lstrip("*")
            t = t.replace("*", "").strip()
            arr = re.match(r"(\w+)\[(\w+)\]", name)
            dim = None
            if arr:
                name, dim = arr.groups()
            fields.append((name, t, ptr, dim))
        out[m.group(1)] = fields
    return out


def rust_structs() -> dict:
    out = {}
    for m in re.finditer(r"pub struct (gg_\w+) \{(.*?)\}", SYS, re.S):
        fields = []
        for f in re.finditer(r"pub (\w+): ([^,\n]+),", m.group(2)):
            fields.append((f.group(1), f.group(2).strip()))
        out[m.group(1)] = fields
    return out


def rust_type_of(t: str, ptr: int, dim) -> str:
    base = C2RUST.get(t, t)
    if ptr:
        base = "*mut " + base
    if dim:
        dim = "GG_N_CLASSES" if dim == "GG_N_CLASSES" else dim
        base = f"[{base}; {dim}]"
    return base


def test_every_struct_field_matches_the_header():
    cs, rs = c_structs(), rust_structs()
    assert set(cs) <= set(rs), set(cs) - set(rs)
    for name, fields in cs.items():
        want = [(n, rust_type_of(t, p, d)) for n, t, p, d in fields]
        assert rs[name] == want, name


def ctypes_struct(name: str, rs: dict):
    fields = []
    for fname, t in rs[name]:
        arr = re.match(r"\[(.+); (\w+)\]", t)
        dim = None
        if arr:
            t, dim = arr.groups()
            dim = 6 if dim == "GG_N_CLASSES" else int(dim)
        if t.startswith("*"):
            ct = C.c_void_p
        elif t in RUST2CT:
            ct = RUST2CT[t]
        else:
            ct = ctypes_struct(t, rs)
        fields.append((fname, ct * dim if dim else ct))
    return type(name, (C.Structure,), {"_fields_": fields})


def test_struct_sizes_equal_the_library_s(gglib):
    rs = rust_structs()
    for name in ("gg_metric_t", "gg_camera_t", "gg_disk_t", "gg_integrator_t",
                 "gg_render_opts_t", "gg_ray_out_t", "gg_stats_t", "gg_scene_t", "gg_prim_t"):
        assert C.sizeof(ctypes_struct(name, rs)) == gglib.gg_struct_size(name.encode()), name


def test_every_entry_point_is_declared_with_its_parameters():
    h = strip_comments(HEADER)
    c_fns = {}
    for m in re.finditer(r"GG_API\s+[\w\s\*]+?\b(gg_\w+)\s*\(([^)]*)\)\s*;", h):
        params = m.group(2).strip()
        c_fns[m.group(1)] = 0 if params in ("", "void") else params.count(",") + 1
    r_fns = {}
    for m in re.finditer(r"pub fn (gg_\w+)\(([^)]*)\)", SYS):
        params = m.group(2).strip().rstrip(",")
        r_fns[m.group(1)] = 0 if not params else params.count(",") + 1
    assert len(c_fns) > 30
    assert set(c_fns) == set(r_fns), set(c_fns) ^ set(r_fns)
    for name, n in c_fns.items():
        assert r_fns[name] == n, name


def test_constants_equal_the_header_s():
    defines = dict(re.findall(r"#define (GG_[A-Z0-9_]+) \(?(-?\d+)\)?", HEADER))
    consts = dict(re.findall(r"pub const (GG_[A-Z0-9_]+): \w+ = (-?\d+);", SYS))
    assert len(consts) > 30
    for name, value in consts.items():
        assert defines[name] == value, name
    for name in defines:
        assert name in consts, name


@pytest.mark.parametrize("fn", ["render", "render_with_disk"])
def test_safe_wrapper_keeps_the_reference_signatures(fn):
    # renderer.rs:82-101: (metric, camera[, disk], width, height, opts) -> RgbImage
    disk = "disk: &AccretionDisk,\\s*" if fn == "render_with_disk" else ""
    pat = (rf"pub fn {fn}<M: GpuMetric>\(metric: &M, camera: &Camera,\s*{disk}width: u32, "
           r"height: u32,\s*opts: RenderOptions\)\s*-> RgbImage")
    assert re.search(pat, SAFE), fn
