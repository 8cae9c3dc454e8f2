"""The Rust binding (crates/marl-cuda/src/ffi.rs) against the C header
(include/marl_cuda.h), checked as text: no Rust toolchain is needed.

- every C struct has a #[repr(C)] Rust struct with the same fields, in the
  same order, of the corresponding types (so the two layouts are identical);
- every C entry point is declared in the extern "C" block with the same
  parameter and return types, and the block declares nothing else;
- every constant both sides define has the same value;
- the safe wrapper (src/lib.rs) copies every field of marl_sim_params from
  SimulationConfig.
"""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "marl_cuda.h")
CRATE = os.path.join(ROOT, "crates", "marl-cuda")
FFI = os.path.join(CRATE, "src", "ffi.rs")
LIB = os.path.join(CRATE, "src", "lib.rs")

C_BASE = {"float": "f32", "double": "f64", "int32_t": "i32", "uint32_t": "u32", "uint64_t": "u64",
          "uint16_t": "u16", "uint8_t": "u8", "char": "c_char", "void": "c_void", "marl_status": "Status",
          "size_t": "usize", "int": "i32"}


def rust_name(c_type: str) -> str:
    if c_type in C_BASE:
        return C_BASE[c_type]
    assert c_type.startswith("marl_"), c_type
    return "".join(w.capitalize() for w in c_type[len("marl_"):].split("_"))


def strip_c_comments(s: str) -> str:
    s = re.sub(r"/\*.*?\*/", " ", s, flags=re.S)
    return re.sub(r"//[^\n]*", " ", s)


def c_constants(src: str) -> dict:
    out = {}
    for name, expr in re.findall(r"#define\s+(MARL_\w+)\s+(.+)", src):
        if name == "MARL_CUDA_H":
            continue
        out[name] = eval(expr.strip(), {}, dict(out))
    for body in re.findall(r"enum\s*(?:\w+\s*)?\{(.*?)\}", src, flags=re.S):
        for name, val in re.findall(r"(MARL_\w+)\s*=\s*(\w+)", body):
            out[name] = int(val, 0)
    return out


def c_type_of(decl: str, consts: dict, param: bool) -> str:
    """Rust spelling of one C declaration `const T* name[N]` (name dropped)."""
    decl = decl.strip()
    arr = re.search(r"\[([^\]]*)\]\s*$", decl)
    if arr:
        decl = decl[: arr.start()].strip()
    const = decl.startswith("const ")
    if const:
        decl = decl[len("const "):]
    stars = decl.count("*")
    parts = decl.replace("*", " ").split()
    base = rust_name(parts[0])
    if arr and not param:
        return f"[{base};{eval(arr.group(1), {}, dict(consts))}]"
    if arr and param:  # an array parameter is a pointer
        stars += 1
    t = base
    for i in range(stars):  # `const` qualifies the innermost pointee
        t = ("*const " if (const and i == 0) else "*mut ") + t
    return t.replace(" ", "")


def c_structs(src: str, consts: dict) -> dict:
    out = {}
    for cname, body, tname in re.findall(r"typedef\s+struct\s+(\w+)\s*\{(.*?)\}\s*(\w+)\s*;", src, flags=re.S):
        assert cname == tname
        fields = []
        for stmt in body.split(";"):
            stmt = stmt.strip()
            if not stmt:
                continue
            m = re.match(r"((?:const\s+)?\w+\s*\**)\s*(.*)", stmt, flags=re.S)
            base, rest = m.group(1), m.group(2)
            for d in rest.split(","):
                d = d.strip()
                name = re.match(r"\**\s*(\w+)", d).group(1)
                stars = re.match(r"(\**)", d).group(1)
                fields.append((name, c_type_of(base + stars + " " + d.lstrip("*"), consts, param=False)))
        out[rust_name(cname)] = fields
    return out


def c_functions(src: str, consts: dict) -> dict:
    body = re.sub(r"typedef\s+struct\s+\w+\s*\{.*?\}\s*\w+\s*;", " ", src, flags=re.S)
    body = re.sub(r"typedef[^;]*;", " ", body)
    body = re.sub(r"enum\s*(?:\w+\s*)?\{.*?\}\s*\w*\s*;", " ", body, flags=re.S)
    body = re.sub(r"#[^\n]*", " ", body)
    out = {}
    for ret, name, params in re.findall(r"((?:const\s+)?\w+\s*\**)\s*\b(marl_\w+)\s*\(([^)]*)\)\s*;", body):
        ps = []
        if params.strip() != "void":
            for p in params.split(","):
                p = p.strip()
                m = re.match(r"(.*?)(\w+)(\s*\[[^\]]*\])?$", p, flags=re.S)
                ps.append(c_type_of(m.group(1) + (m.group(3) or ""), consts, param=True))
        r = ret.strip()
        out[name] = (ps, None if r == "void" else c_type_of(r, consts, param=True))
    return out


def rust_norm(t: str, consts: dict) -> str:
    t = re.sub(r"\s+", " ", t.strip())
    t = re.sub(r"\[(\w+);\s*(\w+)\]", lambda m: f"[{m.group(1)};{consts.get(m.group(2), m.group(2))}]", t)
    return t.replace(" ", "").replace("ffi::", "")


def rust_constants(src: str) -> dict:
    out = {}
    for name, expr in re.findall(r"pub const (\w+):\s*\w+\s*=\s*([^;]+);", src):
        out[name] = eval(expr, {}, dict(out))
    return out


def rust_structs(src: str, consts: dict) -> dict:
    out = {}
    for name, body in re.findall(r"#\[repr\(C\)\]\s*(?:#\[[^\]]*\]\s*)*pub struct (\w+)\s*\{(.*?)\n\}", src, flags=re.S):
        out[name] = [(f, rust_norm(t, consts)) for f, t in re.findall(r"pub (\w+):\s*([^,\n]+),", body)]
    return out


def rust_functions(src: str, consts: dict) -> dict:
    block = src[src.index('unsafe extern "C" {'):]
    block = re.sub(r"//[^\n]*", " ", block)
    out = {}
    for name, params, ret in re.findall(r"pub fn (\w+)\((.*?)\)\s*(?:->\s*([^;]+))?;", block, flags=re.S):
        ps = [rust_norm(p.split(":", 1)[1], consts) for p in params.split(",") if p.strip()]
        out[name] = (ps, rust_norm(ret, consts) if ret else None)
    return out


def load():
    with open(HEADER) as f:
        h = strip_c_comments(f.read())
    with open(FFI) as f:
        r = f.read()
    cc = c_constants(h)
    rc = rust_constants(r)
    return h, r, cc, rc


def test_crate_files_exist():
    for p in ("Cargo.toml", "build.rs", "src/ffi.rs", "src/lib.rs"):
        assert os.path.exists(os.path.join(CRATE, p)), p


def test_constants_agree():
    _, _, cc, rc = load()
    common = set(cc) & set(rc)
    assert {"MARL_S_EXT", "MARL_M_INT", "MARL_OK", "MARL_ERR_TIMEOUT", "MARL_EVENT_DEATH",
            "MARL_SURR_PARAMS", "MARL_SOURCES_DIRICHLET"} <= common
    for k in sorted(common):
        assert cc[k] == rc[k], (k, cc[k], rc[k])
    missing = sorted(k for k in cc if k not in rc)
    assert not missing, missing


def test_structs_match_field_for_field():
    h, r, cc, rc = load()
    cs = c_structs(h, cc)
    rs = rust_structs(r, rc)
    assert len(cs) >= 18
    for name, fields in cs.items():
        assert name in rs, f"no #[repr(C)] struct {name} in ffi.rs"
        assert rs[name] == fields, (name, rs[name], fields)
    extra = sorted(set(rs) - set(cs))
    assert not extra, extra


def test_functions_match_signatures():
    h, r, cc, rc = load()
    cf = c_functions(h, cc)
    rf = rust_functions(r, rc)
    assert len(cf) >= 90
    for name, (params, ret) in cf.items():
        assert name in rf, f"{name} not declared in ffi.rs"
        assert rf[name][0] == params, (name, rf[name][0], params)
        assert rf[name][1] == ret, (name, rf[name][1], ret)
    extra = sorted(set(rf) - set(cf))
    assert not extra, extra


def test_exported_symbol_list_matches_header():
    """The ctypes binding's symbol list, which the library-load test checks
    against the built library, names exactly the header's entry points."""
    import sys

    sys.path.insert(0, os.path.join(ROOT, "marl-ochre_b200"))
    import marl_cuda

    h, _, cc, _ = load()
    assert sorted(marl_cuda.EXPORTED) == sorted(c_functions(h, cc))


def test_params_from_copies_every_field():
    h, r, cc, rc = load()
    fields = [f for f, _ in c_structs(h, cc)["SimParams"]]
    with open(LIB) as f:
        lib = f.read()
    body = lib[lib.index("pub fn params_from"):]
    body = body[: body.index("\n}\n")]
    for f in fields:
        assert re.search(rf"\b{f}:", body), f"params_from does not set {f}"
