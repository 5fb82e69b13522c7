"""The Rust FFI crate (rust/spatialrust-cuda-sys/src/lib.rs) against include/srcuda.h.

Rust is not installed here, so the crate cannot be compiled; this test reads
both files as text and fails on any difference a compiler would not catch at
the boundary: a function of the header missing from the crate's extern "C"
block (or the other way round), a parameter or return type that does not map,
a struct whose fields differ in name, order or type, a constant or status
code with another value."""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "srcuda.h")
RUST_SYS = os.path.join(ROOT, "rust", "spatialrust-cuda-sys", "src", "lib.rs")

C_BASE = {
    "float": "f32", "double": "f64", "int": "i32", "char": "c_char", "void": "c_void",
    "uint8_t": "u8", "uint16_t": "u16", "uint32_t": "u32", "uint64_t": "u64",
    "int32_t": "i32", "int64_t": "i64", "size_t": "usize", "srcu_status": "srcu_status",
}
RUST_ALIASES = {"c_int": "i32", "c_uint": "u32", "c_float": "f32", "c_double": "f64"}


def strip_comments(text):
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    return re.sub(r"//[^\n]*", " ", text)


def c_type(base, declarator):
    """Rust spelling of one C declarator: pointee constness decides *const / *mut."""
    toks = base.split()
    const = "const" in toks
    name = [t for t in toks if t not in ("const", "struct")][-1]
    rust = C_BASE.get(name, name)
    m = re.match(r"^\s*((?:\*\s*(?:const\s*)?)*)\s*(\w+)\s*(?:\[(\d+)\])?\s*$", declarator)
    assert m, f"cannot parse declarator {declarator!r}"
    stars = re.findall(r"\*\s*(const)?", m.group(1))
    for star_const in stars:
        rust = ("*const " if const else "*mut ") + rust
        const = bool(star_const)
    if m.group(3):
        rust = f"[{rust}; {m.group(3)}]"
    return m.group(2), rust


def split_decl(decl):
    """'const float *x, *y' -> base 'const float', declarators ['*x', '*y']."""
    decl = " ".join(decl.split())
    first, *rest = decl.split(",")
    m = re.match(r"^(.*?[\w\s]*?)\s*((?:\*\s*(?:const\s*)?)*\w+\s*(?:\[\d+\])?)$", first.strip())
    assert m, f"cannot split {decl!r}"
    base = m.group(1).strip()
    return base, [m.group(2)] + [r.strip() for r in rest]


def parse_header():
    text = strip_comments(open(HEADER).read())
    defines = dict(re.findall(r"#define\s+(SRCU_\w+)\s+(\d+)", text))
    enums = {}
    for body in re.findall(r"typedef\s+enum\s+\w+\s*\{(.*?)\}", text, flags=re.S):
        value = -1
        for item in body.split(","):
            item = item.strip()
            if not item:
                continue
            name, _, v = item.partition("=")
            value = int(v) if v.strip() else value + 1
            enums[name.strip()] = str(value)
    structs = {}
    for name, body in re.findall(r"typedef\s+struct\s+(\w+)\s*\{(.*?)\}\s*\w+\s*;", text, flags=re.S):
        fields = []
        for decl in body.split(";"):
            if not decl.strip():
                continue
            base, decls = split_decl(decl)
            fields += [c_type(base, d) for d in decls]
        structs[name] = fields
    opaque = set(re.findall(r"typedef\s+struct\s+(\w+)\s+\1\s*;", text))
    funcs = {}
    flat = re.sub(r"typedef\s+(struct|enum)\s+\w*\s*\{.*?\}\s*\w+\s*;", " ", text, flags=re.S)
    for ret, name, params in re.findall(
            r"([\w\s\*]+?)\b(srcu_\w+)\s*\(([^;{]*?)\)\s*;", flat, flags=re.S):
        ret = " ".join(ret.split())
        rname, rtype = c_type(ret.replace("*", "").strip() or ret, ("*" * ret.count("*")) + "r")
        params = " ".join(params.split())
        plist = [] if params in ("", "void") else [split_decl(p) for p in params.split(",")]
        funcs[name] = (rtype if ret != "void" else None, [c_type(b, d[0])[1] for b, d in plist])
    return defines, enums, structs, opaque, funcs


def norm_rust(t):
    t = " ".join(t.replace("\n", " ").split())
    t = re.sub(r"\s*;\s*", "; ", t)
    for a, b in RUST_ALIASES.items():
        t = re.sub(rf"\b{a}\b", b, t)
    t = t.replace("* const", "*const").replace("* mut", "*mut")
    return t.strip()


def parse_rust():
    text = re.sub(r"//[^\n]*", " ", open(RUST_SYS).read())
    consts = {k: v for k, v in re.findall(r"pub const (SRCU_\w+)\s*:\s*\w+\s*=\s*(-?\d+)\s*;", text)}
    structs, opaque = {}, set()
    for name, body in re.findall(r"pub struct (\w+)\s*\{(.*?)\}", text, flags=re.S):
        if re.fullmatch(r"\s*_p\s*:\s*\[u8;\s*0\]\s*,?\s*", body):
            opaque.add(name)
            continue
        fields = []
        for f in re.findall(r"pub\s+(\w+)\s*:\s*([^,]+?)\s*(?:,|$)", body.strip() + ","):
            fields.append((f[0], norm_rust(f[1])))
        structs[name] = fields
    block = re.search(r'extern\s+"C"\s*\{(.*)\}', text, flags=re.S).group(1)
    funcs = {}
    for name, params, ret in re.findall(r"pub fn (srcu_\w+)\s*\((.*?)\)\s*(?:->\s*([^;]+))?;", block,
                                        flags=re.S):
        plist = [p for p in (x.strip() for x in params.split(",")) if p]
        funcs[name] = (norm_rust(ret) if ret else None,
                       [norm_rust(p.split(":", 1)[1]) for p in plist])
    aliases = dict(re.findall(r"pub type (\w+)\s*=\s*(\w+)\s*;", text))
    return consts, structs, opaque, funcs, aliases


def test_every_header_function_is_bound_with_matching_types():
    _, _, _, _, cfuncs = parse_header()
    _, _, _, rfuncs, _ = parse_rust()
    assert set(cfuncs) == set(rfuncs), (
        f"missing in Rust: {sorted(set(cfuncs) - set(rfuncs))}; "
        f"not in the header: {sorted(set(rfuncs) - set(cfuncs))}")
    assert len(cfuncs) >= 50
    for name, (cret, cparams) in cfuncs.items():
        rret, rparams = rfuncs[name]
        assert cret == rret, f"{name}: returns {cret} in C, {rret} in Rust"
        assert cparams == rparams, f"{name}: parameters {cparams} in C, {rparams} in Rust"


def test_every_struct_has_the_same_fields_in_the_same_order():
    _, _, cstructs, copaque, _ = parse_header()
    _, rstructs, ropaque, _, _ = parse_rust()
    assert copaque == ropaque, f"opaque types: {copaque} vs {ropaque}"
    assert set(cstructs) == set(rstructs), (
        f"missing in Rust: {sorted(set(cstructs) - set(rstructs))}; "
        f"not in the header: {sorted(set(rstructs) - set(cstructs))}")
    for name, fields in cstructs.items():
        assert fields == rstructs[name], f"struct {name}: {fields} vs {rstructs[name]}"


def test_constants_and_status_codes_have_the_same_values():
    defines, enums, _, _, _ = parse_header()
    consts, _, _, _, aliases = parse_rust()
    want = {**defines, **enums}
    assert want == consts, {k: (want.get(k), consts.get(k)) for k in set(want) | set(consts)
                            if want.get(k) != consts.get(k)}
    assert aliases.get("srcu_status") in ("c_int", "i32")
    assert aliases.get("srcu_kernel_id") in ("c_int", "i32")


def test_safe_wrapper_uses_only_bound_functions():
    _, _, _, rfuncs, _ = parse_rust()
    for rel in ("rust/spatialrust-gpu-cuda/src/lib.rs",):
        text = open(os.path.join(ROOT, rel)).read()
        used = set(re.findall(r"sys::(srcu_\w+)\s*\(", text))
        assert used and used <= set(rfuncs), sorted(used - set(rfuncs))
