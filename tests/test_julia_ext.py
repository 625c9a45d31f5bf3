"""Static checks of the Julia extension (frequencydriftratetransforms.jl_b200/julia/
B200FrequencyDriftRateTransformsExt.jl) against the C ABI it binds (include/fdr_b200.h).

Julia is not installed here, so the module cannot be loaded; these checks read it as text:
every ccall names a symbol the header declares, with as many argument types as the C
prototype has parameters and Julia types that match the C types (scalars by width and kind,
pointers by depth and pointee); the mirrored C structs have the C field types in order; and
the module's blocks are balanced."""
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
JL = os.path.join(ROOT, "frequencydriftratetransforms.jl_b200", "julia",
                  "B200FrequencyDriftRateTransformsExt.jl")
HDR = os.path.join(ROOT, "include", "fdr_b200.h")

# C scalar type -> Julia names accepted for it
SCALARS = {
    "int": {"Cint", "Int32"}, "int32_t": {"Int32", "Cint"}, "int64_t": {"Int64"},
    "uint32_t": {"UInt32", "Cuint"}, "uint64_t": {"UInt64"}, "float": {"Float32", "Cfloat"},
    "double": {"Float64", "Cdouble"}, "char": {"UInt8", "Cchar"},
}
STRUCTS = {"fdr_zdt_info": "ZDTInfo", "fdr_batch_channel": "BatchChannel",
           "fdr_hit_cluster": "HitCluster"}
OPAQUE = {"fdr_zdt", "fdr_batch", "fdr_propose_net", "fdr_fft_ws", "void", "CUstream_st"}


def _strip_c_comments(s):
    return re.sub(r"/\*.*?\*/", "", s, flags=re.S)


def c_prototypes():
    s = _strip_c_comments(open(HDR).read())
    protos = {}
    for m in re.finditer(r"^([A-Za-z_][\w\s\*]*?)\b(fdr_\w+)\s*\(([^)]*)\)\s*;", s, flags=re.M):
        ret, name, params = m.group(1).strip(), m.group(2), m.group(3).strip()
        plist = [] if params in ("", "void") else [p.strip() for p in params.split(",")]
        protos[name] = (ret, plist)
    return protos


def c_structs():
    """name -> [(field, base type, pointer depth, array length or 0)] of the header's
    typedef'd structs (declarations of the form `type a, *b, c[8];`)."""
    s = _strip_c_comments(open(HDR).read())
    out = {}
    for m in re.finditer(r"typedef struct (\w+) \{(.*?)\} \1;", s, flags=re.S):
        fields = []
        for decl in m.group(2).split(";"):
            toks = [t for t in decl.replace("*", " * ").replace(",", " , ").split() if t != "const"]
            if not toks:
                continue
            base, rest = toks[0], " ".join(toks[1:])
            for item in rest.split(","):
                depth = item.count("*")
                name = item.replace("*", "").strip()
                arr = re.match(r"(\w+)\[(\d+)\]", name)
                if arr:
                    fields.append((arr.group(1), base, depth, int(arr.group(2))))
                else:
                    fields.append((name, base, depth, 0))
        out[m.group(1)] = fields
    return out


def c_type(param):
    """(base, depth) of a C parameter or return type (names and const stripped)."""
    p = param.replace("*", " * ")
    toks = [t for t in p.split() if t != "const"]
    depth = toks.count("*")
    toks = [t for t in toks if t != "*"]
    if toks and toks[0] == "fdr_stream_t":
        return "CUstream_st", depth + 1
    base = toks[0]
    return base, depth


def _split_top(s, sep=","):
    out, depth, cur = [], 0, ""
    for ch in s:
        if ch in "({[":
            depth += 1
        elif ch in ")}]":
            depth -= 1
        if ch == sep and depth == 0:
            out.append(cur.strip())
            cur = ""
        else:
            cur += ch
    if cur.strip():
        out.append(cur.strip())
    return out


def _balanced(s, i):
    """Index just past the bracket group that opens at s[i]."""
    pairs = {"(": ")", "{": "}", "[": "]"}
    stack = [pairs[s[i]]]
    j = i + 1
    while stack:
        ch = s[j]
        if ch in pairs:
            stack.append(pairs[ch])
        elif ch in ")}]":
            assert ch == stack.pop(), f"unbalanced bracket at {j}"
        elif ch == '"':
            j += 1
            while s[j] != '"':
                j += 2 if s[j] == "\\" else 1
        j += 1
    return j


def julia_ccalls():
    src = _julia_code(open(JL).read())
    calls = []
    for m in re.finditer(r"ccall\(\(:(\w+),\s*libfdrb200\),", src):
        start = src.index("(", m.start())
        end = _balanced(src, start)
        inner = src[start + 1:end - 1]
        parts = _split_top(inner)
        name = m.group(1)
        ret = parts[1]
        argt = parts[2]
        assert argt.startswith("(") and argt.endswith(")"), (name, argt)
        types = _split_top(argt[1:-1])
        nargs = len(parts) - 3
        calls.append((name, ret, types, nargs))
    return calls


def _julia_code(s):
    """The source with comments removed and string contents blanked."""
    out, i = [], 0
    while i < len(s):
        ch = s[i]
        if ch == "#":
            while i < len(s) and s[i] != "\n":
                i += 1
            continue
        if ch == '"':
            j = i + 1
            while s[j] != '"':
                j += 2 if s[j] == "\\" else 1
            out.append('""')
            i = j + 1
            continue
        out.append(ch)
        i += 1
    return "".join(out)


def julia_type(t):
    """(base, depth) of a Julia ccall type: Ptr/CuPtr/Ref add a level of indirection."""
    t = t.strip()
    depth = 0
    while True:
        m = re.match(r"^(Ptr|CuPtr|Ref)\{(.+)\}$", t)
        if not m:
            break
        depth += 1
        t = m.group(2).strip()
    if t == "Cstring":
        return "Cchar", depth + 1
    return t, depth


def _compatible(cbase, cdepth, jbase, jdepth):
    if cdepth != jdepth:
        return False
    if cbase in SCALARS:
        return jbase in SCALARS[cbase]
    if cbase in STRUCTS:
        return jbase in (STRUCTS[cbase], "Cvoid")
    if cbase in OPAQUE:
        return jbase == "Cvoid"
    return False


def test_every_ccall_matches_a_declared_prototype():
    protos = c_prototypes()
    calls = julia_ccalls()
    assert len(calls) >= 25
    seen = set()
    for name, ret, types, nargs in calls:
        assert name in protos, f"{name} is not declared in include/fdr_b200.h"
        cret, cparams = protos[name]
        assert len(types) == len(cparams), (name, types, cparams)
        assert nargs == len(types), f"{name}: {nargs} arguments for {len(types)} types"
        rb, rd = c_type(cret)
        jb, jd = julia_type(ret)
        assert _compatible(rb, rd, jb, jd), (name, cret, ret)
        for cp, jt in zip(cparams, types):
            cb, cd = c_type(cp)
            jb, jd = julia_type(jt)
            # a pointer to a pointer (fdr_zdt**, float* const*) is passed as
            # Ref{Ptr{Cvoid}} / Ptr{CuPtr{Float32}}: compare the innermost pointee
            assert _compatible(cb, cd, jb, jd), f"{name}: C `{cp}` vs Julia `{jt}`"
        seen.add(name)
    # the reference API the extension forwards reaches these entry points
    for needed in ["fdr_zdt_create", "fdr_zdt_destroy", "fdr_zdt_get_info", "fdr_zdt_buffers",
                   "fdr_zdt_input", "fdr_zdt_preprocess", "fdr_zdt_convolve",
                   "fdr_zdt_postprocess", "fdr_zdt_output", "fdr_zdt_execute",
                   "fdr_zdtfdr_protohits", "fdr_intshift", "fdr_intfdr_shifts",
                   "fdr_fftfdr_workspace", "fdr_fftfdr_workspace_update", "fdr_fftfdr_destroy",
                   "fdr_fftfdr_rfft_buffer", "fdr_fdshiftsum", "fdr_fdshift", "fdr_fftfdr",
                   "fdr_stats", "fdr_normalize", "fdr_findprotohits", "fdr_synchronize",
                   "fdr_last_error_string", "fdr_taylor_tree"]:
        assert needed in seen, needed


def test_mirrored_structs_match_the_header():
    src = _julia_code(open(JL).read())
    m = re.search(r"struct ZDTInfo\n(.*?)\nend", src, flags=re.S)
    assert m
    jfields = []
    for line in m.group(1).splitlines():
        line = line.strip()
        if line:
            n, t = line.split("::")
            jfields.append((n.strip(), t.strip()))
    cfields = c_structs()["fdr_zdt_info"]
    flat = []
    for name, base, depth, arr in cfields:
        flat.append((name, base, arr))
    assert len(flat) == len(jfields), (flat, jfields)
    for (cn, cb, arr), (jn, jt) in zip(flat, jfields):
        if arr:
            assert jt == f"NTuple{{{arr},{next(iter(sorted(SCALARS[cb])))}}}" or \
                jt in {f"NTuple{{{arr},{x}}}" for x in SCALARS[cb]}, (cn, jt)
        else:
            assert jt in SCALARS[cb], (cn, cb, jt)


def test_method_signatures_cover_the_reference_call_forms():
    """The dispatch fixes a Julia binding needs (zdtfdr.jl:349-421, :297-321): Val window
    methods, a dest::AbstractMatrix method on the B200 workspace (resolving the reference's
    matrix-dest method against the iterable one), the no-dest and allocating forms, show and
    sizeof, and no redefinition of the reference CUDA extension's fdrsynchronize method."""
    src = _julia_code(open(JL).read())
    for pat in [r"window_args\(::Val\{:rect\}", r"window_args\(::Val\{:hamming\}",
                r"window_args\(::Val\{S\}, ws\) where \{S\}",
                r"postprocess!\(w::Val\{:hamming\}, ws::B200ZDTWorkspace\)",
                r"postprocess!\(w::Val\{:rect\}, ws::B200ZDTWorkspace\)",
                r"postprocess!\(::Val\{S\}, ws::B200ZDTWorkspace\) where \{S\}",
                r"function zdtfdr!\(w::Union\{Function,Symbol,Val\}, dests, ws::B200ZDTWorkspace",
                r"function zdtfdr!\(w::Union\{Function,Symbol,Val\}, dest::AbstractMatrix\{<:Real\},\s*ws::B200ZDTWorkspace",
                r"function zdtfdr!\(w::Union\{Function,Symbol,Val\}, ws::B200ZDTWorkspace, spectrogram=nothing",
                r"zdtfdr!\(ws::B200ZDTWorkspace, spectrogram=nothing",
                r"function zdtfdr\(w::Union\{Function,Symbol,Val\}, ws::B200ZDTWorkspace",
                r"zdtfdr\(ws::B200ZDTWorkspace, spectrogram=nothing",
                r"function preprocess!\(ws::B200ZDTWorkspace, r0::Float32=ws.r0\)",
                r"preprocess!\(ws::B200ZDTWorkspace, r0::Real\)",
                r"function Base\.show\(io::IO, ws::B200ZDTWorkspace\)",
                r"function Base\.sizeof\(ws::B200ZDTWorkspace\)",
                r"function fdrsynchronize\(::Type\{<:CuArray\{Float32\}\}\)"]:
        assert re.search(pat, src), pat
    assert not re.search(r"fdrsynchronize\(::Type\{<:CuArray\}\)", src)
    assert "workspace.Ys" not in src


def test_blocks_balance():
    src = _julia_code(open(JL).read())
    # `end` inside brackets is an index (a[end]); block keywords open at statement level
    depth_br, opens, ends = 0, 0, 0
    for tok in re.finditer(r"[\[\](){}]|\b(function|struct|mutable struct|module|if|for|while|"
                           r"let|begin|do|try|quote|macro|end)\b", src):
        t = tok.group(0)
        if t in "[({":
            depth_br += 1
        elif t in "])}":
            depth_br -= 1
        elif t == "end":
            if depth_br == 0:
                ends += 1
        elif depth_br == 0 or t == "do":
            if t == "struct" and src[max(0, tok.start() - 8):tok.start()] == "mutable ":
                continue
            opens += 1
    # one-line definitions `f(x) = ...` open nothing; `function` always opens a block
    assert depth_br == 0
    assert opens == ends, (opens, ends)
