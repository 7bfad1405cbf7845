"""The Rust FFI crate (shallow-water_b200/rust/shallow-water-cuda-sys) against the
C header it binds: every entry point of include/sw_cuda.h is declared in the
crate's extern block with the same argument count and pointer/value kinds, and
the crate's constants equal the header's.  No Rust toolchain is needed: the
crate source is parsed as text."""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "sw_cuda.h")
SYS = os.path.join(ROOT, "shallow-water_b200", "rust", "shallow-water-cuda-sys", "src", "lib.rs")
SAFE = os.path.join(ROOT, "shallow-water_b200", "rust", "shallow-water-cuda", "src")


def _c_prototypes():
    text = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    out = {}
    for ret, name, args in re.findall(r"^\s*((?:const\s+)?[a-z_ ]+\**)\s*(sw_[a-z0-9_]+)\s*\(([^)]*)\)\s*;",
                                      text, flags=re.M):
        args = args.strip()
        params = [] if args in ("", "void") else [a.strip() for a in args.split(",")]
        kinds = ["ptr" if ("*" in a or "[" in a) else "val" for a in params]
        out[name] = (ret.strip(), kinds)
    return out


def _rust_externs():
    text = open(SYS).read()
    block = re.search(r'extern "C" \{(.*)\}', text, flags=re.S).group(1)
    out = {}
    for name, args, ret in re.findall(r"pub fn (sw_[a-z0-9_]+)\(([^)]*)\)\s*(->\s*[^;]+)?;", block):
        params = [a.strip() for a in args.split(",") if a.strip()]
        kinds = ["ptr" if "*" in a.split(":", 1)[1] else "val" for a in params]
        out[name] = ((ret or "").replace("->", "").strip(), kinds)
    return out


def test_every_header_entry_point_is_bound_with_matching_arguments():
    c = _c_prototypes()
    r = _rust_externs()
    assert len(c) >= 50
    assert sorted(c) == sorted(r), "header-only: %s, crate-only: %s" % (sorted(set(c) - set(r)), sorted(set(r) - set(c)))
    for name, (cret, ckinds) in c.items():
        rret, rkinds = r[name]
        assert ckinds == rkinds, "%s: C %s vs Rust %s" % (name, ckinds, rkinds)
        assert (cret == "void") == (rret == ""), name


def test_constants_match_header():
    text = open(HEADER).read()
    defines = {k: int(v) for k, v in re.findall(r"#define (SW_[A-Z0-9_]+) (\d+)", text)}
    enum = re.search(r"enum sw_field \{(.*?)\};", text, flags=re.S).group(1)
    names = [n.strip().split("=")[0].strip() for n in enum.replace("\n", " ").split(",") if n.strip()]
    defines.update({n: i for i, n in enumerate(names)})
    rs = {k: int(v) for k, v in re.findall(r"pub const (SW_[A-Z0-9_]+): c_int = (\d+);", open(SYS).read())}
    assert rs, "no constants found in the crate"
    for k, v in rs.items():
        assert defines.get(k) == v, "%s: crate %d, header %s" % (k, v, defines.get(k))
    for k in ("SW_OK", "SW_FP64", "SW_MIXED", "SW_FP32", "SW_ERR_PSOLVE_DIVERGED", "SW_GS", "SW_NFIELDS"):
        assert k in rs, k


def test_safe_crate_keeps_reference_names_and_calls_only_bound_symbols():
    src = "".join(open(os.path.join(SAFE, f)).read() for f in sorted(os.listdir(SAFE)) if f.endswith(".rs"))
    for name in ("pub fn forfft", "pub fn revfft", "pub fn initfft", "pub fn factorisen", "pub struct D2FFT",
                 "pub fn ptospc", "pub fn spctop", "pub fn xderiv", "pub fn yderiv", "pub struct Spectral",
                 "pub fn main_invert", "pub fn jacob", "pub fn divs", "pub fn ptospc3d", "pub fn spctop3d",
                 "pub fn deal3d", "pub fn deal2d", "pub fn spec1d", "pub struct State", "pub fn advance",
                 "pub fn psolve", "pub fn source", "pub fn vertical", "pub fn coeffs", "pub fn cpsource"):
        assert name in src, name
    bound = set(_rust_externs())
    used = set(re.findall(r"sys::(sw_[a-z0-9_]+)\(", src))
    assert used and used <= bound, sorted(used - bound)
