"""The Rust `-sys` crate (crates/wavecore-b200-sys/src/lib.rs) against include/wavecore_c.h, CPU only.

No Rust toolchain exists here, so the binding is checked by reading both files: every function of
the header is declared in the crate's `extern "C"` block with the same parameter names and types
(C types mapped to their Rust equivalents, pointer constness included) and the same return type,
and nothing else is; every struct has the same fields in the same order with the same types; every
status, order and preconditioner constant has the same value.
"""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "wavecore_c.h")
CRATE = os.path.join(ROOT, "crates", "wavecore-b200-sys", "src", "lib.rs")

BASE = {"uint64_t": "u64", "int32_t": "i32", "uint32_t": "u32", "uint8_t": "u8", "double": "f64",
        "float": "f32", "void": "c_void", "char": "c_char", "size_t": "usize"}


def strip_c_comments(s):
    s = re.sub(r"/\*.*?\*/", " ", s, flags=re.S)
    return re.sub(r"//[^\n]*", " ", s)


def rust_of_c_type(ctype):
    """Rust spelling of a C type such as `const double* const*` or `wc_solver**`."""
    t = ctype.replace("*", " * ").split()
    stars = [k for k, tok in enumerate(t) if tok == "*"]
    base_tokens = [tok for tok in t[: stars[0]] if tok != "const"] if stars else [tok for tok in t if tok != "const"]
    assert len(base_tokens) == 1, ctype
    base = BASE.get(base_tokens[0], base_tokens[0])
    if not stars:
        return base
    out = base
    for n, pos in enumerate(stars):
        # constness of this pointer's pointee: a qualifier between the previous star and this one
        prev = stars[n - 1] + 1 if n > 0 else 0
        const = "const" in t[prev:pos]
        out = ("*const " if const else "*mut ") + out
    return out


def c_functions():
    text = strip_c_comments(open(HEADER).read())
    text = re.sub(r"#[^\n]*", " ", text)
    text = re.sub(r"typedef\s+(struct|enum)[^;]*?\{.*?\}\s*\w+\s*;", " ", text, flags=re.S)
    text = re.sub(r"typedef\s+struct\s+\w+\s+\w+\s*;", " ", text)
    out = {}
    for m in re.finditer(r"([\w\s\*]+?)\b(wc_\w+)\s*\(([^)]*)\)\s*;", text):
        ret = " ".join(m.group(1).split())
        name = m.group(2)
        params = []
        args = m.group(3).strip()
        if args and args != "void":
            for a in args.split(","):
                a = " ".join(a.split())
                arr = re.match(r"(.*?)\s*\[[^\]]*\]$", a)
                if arr:
                    pm = re.match(r"(.*?)(\w+)$", arr.group(1))
                    ptype, pname = pm.group(1).strip() + "*", pm.group(2)
                else:
                    pm = re.match(r"(.*?)(\w+)$", a)
                    ptype, pname = pm.group(1).strip(), pm.group(2)
                params.append((pname, rust_of_c_type(ptype)))
        out[name] = (params, None if ret == "void" else rust_of_c_type(ret))
    return out


def c_structs():
    text = strip_c_comments(open(HEADER).read())
    out = {}
    for m in re.finditer(r"typedef\s+struct\s+(\w+)\s*\{(.*?)\}\s*(\w+)\s*;", text, flags=re.S):
        fields = []
        for decl in m.group(2).split(";"):
            decl = " ".join(decl.split())
            if not decl:
                continue
            dm = re.match(r"((?:const\s+)?\w+\**)\s*(.*)$", decl)
            ctype, names = dm.group(1), dm.group(2)
            for nm in names.split(","):
                nm = nm.strip()
                fields.append((nm.strip("* "), rust_of_c_type(ctype + "*" * nm.count("*"))))
        out[m.group(3)] = fields
    return out


def c_constants():
    text = strip_c_comments(open(HEADER).read())
    vals = {k: int(v) for k, v in re.findall(r"\b(WC_[A-Z0-9_]+)\s*=\s*(\d+)", text)}
    vals.update({k: int(v) for k, v in re.findall(r"#define\s+(WC_[A-Z0-9_]+)\s+(\d+)", text)})
    return vals


def rust_functions():
    text = open(CRATE).read()
    block = text[text.index('extern "C" {'):]
    out = {}
    for m in re.finditer(r"pub fn (\w+)\s*\((.*?)\)\s*(->\s*([^;]+))?;", block, flags=re.S):
        params = []
        for a in m.group(2).split(","):
            a = " ".join(a.split())
            if not a:
                continue
            n, t = a.split(":", 1)
            params.append((n.strip(), " ".join(t.split())))
        out[m.group(1)] = (params, " ".join(m.group(4).split()) if m.group(4) else None)
    return out


def rust_structs():
    text = open(CRATE).read()
    out = {}
    for m in re.finditer(r"pub struct (\w+)\s*\{(.*?)\}", text, flags=re.S):
        fields = []
        for line in m.group(2).split(","):
            fm = re.match(r"pub (\w+): (.+)$", " ".join(line.split()))
            if fm:
                fields.append((fm.group(1), fm.group(2)))
        out[m.group(1)] = fields
    return out


def rust_constants():
    text = open(CRATE).read()
    return {k: int(v) for k, v in re.findall(r"pub const (WC_[A-Z0-9_]+): \w+ = (\d+);", text)}


def test_every_function_of_the_header_is_bound_with_the_same_signature():
    cf, rf = c_functions(), rust_functions()
    assert len(cf) >= 60
    assert set(cf) == set(rf), (sorted(set(cf) - set(rf)), sorted(set(rf) - set(cf)))
    for name, (params, ret) in cf.items():
        rparams, rret = rf[name]
        assert rparams == params, (name, params, rparams)
        assert rret == ret, (name, ret, rret)


def test_every_struct_has_the_same_fields_in_the_same_order():
    cs, rs = c_structs(), rust_structs()
    assert len(cs) >= 12
    for name, fields in cs.items():
        assert name in rs, name
        assert rs[name] == fields, (name, fields, rs[name])


def test_constants_agree():
    cc, rc = c_constants(), rust_constants()
    for name in ("WC_OK", "WC_EINVAL", "WC_EPERIODIC", "WC_ENAN", "WC_EUNCONVERGED", "WC_ETIMEOUT", "WC_ECUDA",
                 "WC_ENOMEM", "WC_EUNSUPPORTED", "WC_ORDER_FIRST", "WC_ORDER_SECOND", "WC_ORDER_FIFTH",
                 "WC_PC_JACOBI", "WC_PC_LEARNED", "WC_GHOST", "WC_KERNEL_KINDS"):
        assert cc[name] == rc[name], name
