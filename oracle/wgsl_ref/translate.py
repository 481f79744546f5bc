"""ORACLE — test infrastructure only.

Mechanical WGSL -> C++ translation of the reference's compute shaders, so that the
reference's own shader source runs on the CPU as the parity pin of the oracle.

Reads (at build time, never at test or bench time):
  src/util.js            uniform field list (uni.addUniform / graphUni.addUniform, util.js:1-35)
  src/main.js            workgroup override values (main.js:34, 181-184)
  src/shaders/ausm.js    solver shaders
  src/shaders/grid.js    grid generation / metric shaders
  src/shaders/graphs.js  force shaders
The shader text is a JS template literal; `${...}` expressions (ternaries on the
template's parameters, calls to other templates, uni.uniformStruct) are evaluated
here.  The WGSL is then rewritten token by token: declarations (let/var/fn/override/
bindings) take C++ form, float literals get an `f` suffix (WGSL abstract floats in an
f32 context), multi-letter swizzles become accessor calls, bindings are qualified so
a local `let x = textureLoad(x, ...)` still reads the binding, WGSL switch cases get
explicit breaks, and shaders with workgroupBarrier() become coroutines.  Nothing of
the translation is committed: build_ref.py writes it under oracle/_ref/.
"""
from __future__ import annotations

import re
import sys
from pathlib import Path

# ----------------------------------------------------------------------------
# 1. JS side: template extraction and evaluation
# ----------------------------------------------------------------------------

_TEMPLATE_DEF = re.compile(r"const\s+(\w+)\s*=\s*(?:\(([^)]*)\)\s*=>\s*)?/\*\s*wgsl\s*\*/\s*`")
_CALL_DEF = re.compile(r"const\s+(\w+)\s*=\s*(\w+)\(([^)]*)\)\s*;")


def _scan_template(text: str, i: int):
    """Parse a template literal body starting after its opening backtick."""
    parts = []
    buf = []
    while True:
        c = text[i]
        if c == "`":
            parts.append(("s", "".join(buf)))
            return parts, i + 1
        if c == "\\":
            buf.append(text[i + 1])
            i += 2
            continue
        if c == "$" and text[i + 1] == "{":
            parts.append(("s", "".join(buf)))
            buf = []
            depth = 1
            j = i + 2
            quote = None
            while depth:
                d = text[j]
                if quote:
                    if d == quote:
                        quote = None
                elif d in "\"'":
                    quote = d
                elif d == "{":
                    depth += 1
                elif d == "}":
                    depth -= 1
                j += 1
            parts.append(("e", text[i + 2 : j - 1]))
            i = j
            continue
        buf.append(c)
        i += 1


class Templates:
    def __init__(self):
        self.defs = {}   # name -> (params[(name, default)], parts)
        self.calls = {}  # name -> (func, argtext)

    def load(self, path: Path):
        text = path.read_text()
        for m in _TEMPLATE_DEF.finditer(text):
            params = []
            if m.group(2) is not None:
                for p in m.group(2).split(","):
                    p = p.strip()
                    if not p:
                        continue
                    if "=" in p:
                        n, d = p.split("=", 1)
                        params.append((n.strip(), d.strip()))
                    else:
                        params.append((p, None))
            parts, _ = _scan_template(text, m.end())
            self.defs[m.group(1)] = (params, parts)
        for m in _CALL_DEF.finditer(text):
            if m.group(2) in self.defs:
                self.calls[m.group(1)] = (m.group(2), m.group(3))

    # -- a tiny evaluator for the JS expressions that occur inside ${...} --
    def _tokens(self, s):
        return re.findall(r'"[^"]*"|\'[^\']*\'|==|!=|[A-Za-z_]\w*(?:\.\w+)*|\d+(?:\.\d+)?|[()?:,]', s)

    def _eval(self, toks, env):
        val, rest = self._ternary(toks, env)
        return val, rest

    def _ternary(self, toks, env):
        cond, toks = self._equality(toks, env)
        if toks and toks[0] == "?":
            a, toks = self._ternary(toks[1:], env)
            assert toks[0] == ":", toks
            b, toks = self._ternary(toks[1:], env)
            return (a if cond else b), toks
        return cond, toks

    def _equality(self, toks, env):
        a, toks = self._primary(toks, env)
        while toks and toks[0] in ("==", "!="):
            op = toks[0]
            b, toks = self._primary(toks[1:], env)
            a = (a == b) if op == "==" else (a != b)
        return a, toks

    def _primary(self, toks, env):
        t = toks[0]
        if t == "(":
            v, toks = self._ternary(toks[1:], env)
            assert toks[0] == ")"
            return v, toks[1:]
        if t[0] in "\"'":
            return t[1:-1], toks[1:]
        if t[0].isdigit():
            return (float(t) if "." in t else int(t)), toks[1:]
        if t in ("true", "false"):
            return t == "true", toks[1:]
        if len(toks) > 1 and toks[1] == "(":  # template call
            args = []
            toks = toks[2:]
            while toks[0] != ")":
                v, toks = self._ternary(toks, env)
                args.append(v)
                if toks[0] == ",":
                    toks = toks[1:]
            return self.expand(t, args), toks[1:]
        if t in env:
            return env[t], toks[1:]
        if t in ("uni.uniformStruct",):
            return "\n/*@UNIFORMS@*/\n", toks[1:]
        if t in ("graphUni.uniformStruct",):
            return "\n/*@GRAPHUNIFORMS@*/\n", toks[1:]
        raise KeyError(f"unknown JS name in template: {t}")

    def expand(self, name, args=()):
        if name in self.calls:
            fn, argtext = self.calls[name]
            vals = []
            toks = self._tokens(argtext)
            while toks:
                v, toks = self._ternary(toks, {})
                vals.append(v)
                if toks and toks[0] == ",":
                    toks = toks[1:]
            return self.expand(fn, vals)
        params, parts = self.defs[name]
        env = {}
        for k, (pn, dflt) in enumerate(params):
            if k < len(args):
                env[pn] = args[k]
            else:
                v, _ = self._ternary(self._tokens(dflt), {})
                env[pn] = v
        out = []
        for kind, s in parts:
            if kind == "s":
                out.append(s)
            else:
                v, rest = self._ternary(self._tokens(s), env)
                assert not rest, (s, rest)
                out.append(str(v) if not isinstance(v, bool) else ("true" if v else "false"))
        return "".join(out)


def uniform_fields(util_js: str, var: str):
    """Field list of a uniform struct from `<var>.addUniform("name", "type")` calls."""
    return re.findall(rf'\b{var}\.addUniform\("(\w+)",\s*"(\w+)"\)', util_js)


def workgroup_overrides(main_js: str):
    m = re.search(r"const\s*\[\s*wg_x\s*,\s*wg_y\s*\]\s*=\s*\[\s*(\d+)\s*,\s*(\d+)\s*\]", main_js)
    return {"WG_X": int(m.group(1)), "WG_Y": int(m.group(2))}


# ----------------------------------------------------------------------------
# 2. WGSL -> C++
# ----------------------------------------------------------------------------

_TOK = re.compile(
    r"\s+|[A-Za-z_]\w*|(?:\d+\.\d*|\.\d+|\d+)(?:[eE][+-]?\d+)?[uif]?|>>=|<<=|->|==|!=|<=|>=|&&|\|\||\+=|-=|\*=|/=|%=|>>|<<|.",
    re.S,
)
_SWIZZLE = re.compile(r"^(?:[xyzw]{2,4}|[rgba]{2,4})$")


def strip_comments(src: str) -> str:
    src = re.sub(r"/\*(?!@).*?\*/", " ", src, flags=re.S)
    src = re.sub(r"//[^\n]*", "", src)
    return src


def tokenize(src: str):
    return _TOK.findall(src)


def is_ws(t):
    return t.isspace()


def fix_number(t):
    if re.fullmatch(r"(?:\d+\.\d*|\.\d+|\d+)(?:[eE][+-]?\d+)?", t) and ("." in t or "e" in t.lower()):
        return t + "f"
    if t.endswith("f") and re.fullmatch(r"[\d.eE+-]+f", t):
        return t
    if t.endswith("i"):
        return t[:-1]
    return t


_CTYPE = {
    "f32": "f32", "u32": "u32", "i32": "i32", "bool": "bool",
    "vec2f": "vec2f", "vec3f": "vec3f", "vec4f": "vec4f",
    "vec2u": "vec2u", "vec3u": "vec3u", "vec4u": "vec4u",
    "vec2i": "vec2i", "vec3i": "vec3i", "vec4i": "vec4i",
}


class Module:
    def __init__(self, name, wgsl, overrides, uni_fields, guni_fields):
        self.name = name
        self.src = strip_comments(wgsl)
        self.overrides = overrides
        self.uni_fields = uni_fields
        self.guni_fields = guni_fields
        self.bindings = []        # (index, kind, name, ctype)
        self.globals = set()
        self.workgroup_vars = []  # (name, ctype, size_expr)
        self.wgsize = None
        self.builtins = []        # builtin names in main's parameter order
        self.barrier = "workgroupBarrier" in self.src

    # -- helpers over token lists --
    @staticmethod
    def _skip_ws(toks, i):
        while i < len(toks) and is_ws(toks[i]):
            i += 1
        return i

    def _until(self, toks, i, stop):
        """Collect tokens until the top-level token `stop` (not consumed)."""
        depth = 0
        out = []
        while True:
            t = toks[i]
            if depth == 0 and t == stop:
                return out, i
            if t in "([{":
                depth += 1
            elif t in ")]}":
                depth -= 1
            out.append(t)
            i += 1

    def _type_text(self, toks):
        return "".join(t for t in toks if not is_ws(t)).strip()

    def _ctype(self, wtype):
        wtype = wtype.replace(" ", "")
        if wtype in _CTYPE:
            return _CTYPE[wtype]
        if wtype in ("Uniforms", "GraphUniforms"):
            return wtype
        m = re.fullmatch(r"array<(\w+)>", wtype)
        if m:
            return f"Storage<{_CTYPE[m.group(1)]}>"
        if wtype == "atomic<u32>":
            return "AtomicU32"
        if wtype == "texture_2d<f32>":
            return "TexF"
        if wtype == "texture_2d<i32>":
            return "TexI"
        if wtype.startswith("texture_storage_2d<"):
            return "TexW"
        raise ValueError(f"{self.name}: unsupported WGSL type {wtype}")

    # -- body translation --
    def _body(self, toks):
        out = []
        shadow = []  # (name, depth)
        depth = 0
        i = 0
        n = len(toks)
        prev_sig = None
        in_switch = []

        def sig_prev():
            for t in reversed(out):
                if not is_ws(t):
                    return t
            return None

        while i < n:
            t = toks[i]
            if is_ws(t):
                out.append(t)
                i += 1
                continue
            if t == "{":
                depth += 1
                out.append(t)
                i += 1
                continue
            if t == "}":
                depth -= 1
                shadow = [s for s in shadow if s[1] <= depth]
                if in_switch and depth < in_switch[-1]:
                    in_switch.pop()
                out.append(t)
                i += 1
                continue
            if t == "switch":
                # remember the depth of the switch's own brace block
                in_switch.append(depth + 1)
                out.append(t)
                i += 1
                continue
            if t in ("case", "default") and in_switch:
                if sig_prev() == "}":
                    out.append(" break; ")
                if t == "case":
                    j = self._skip_ws(toks, i + 1)
                    labels, j = self._until(toks, j, ":")
                    labs = [x.strip() for x in "".join(labels).split(",") if x.strip()]
                    out.append(" ".join(f"case {fix_number(l)}:" for l in labs))
                    i = j + 1
                else:
                    out.append("default")
                    i += 1
                continue
            if t in ("let", "var"):
                j = self._skip_ws(toks, i + 1)
                if toks[j] == "<":  # var<function> etc.
                    _, j = self._until(toks, j, ">")
                    j = self._skip_ws(toks, j + 1)
                name = toks[j]
                j = self._skip_ws(toks, j + 1)
                ctype = None
                if toks[j] == ":":
                    j = self._skip_ws(toks, j + 1)
                    ty = []
                    while toks[j] not in ("=", ";"):
                        ty.append(toks[j])
                        j += 1
                    ctype = self._ctype(self._type_text(ty))
                if toks[j] == "=":
                    init, k = self._until(toks, j + 1, ";")
                    init_c = self._expr(init, shadow)
                    decl = ("const " if t == "let" else "") + (ctype or "auto")
                    out.append(f"{decl} {name} ={init_c};")
                    i = k + 1
                else:  # var NAME: T;
                    out.append(f"{ctype} {name}{{}};")
                    i = j + 1
                if name in self.globals:
                    shadow.append((name, depth))
                continue
            if t == "workgroupBarrier":
                j = self._skip_ws(toks, i + 1)
                assert toks[j] == "("
                _, j = self._until(toks, j + 1, ")")
                j = self._skip_ws(toks, j + 1)
                if toks[j] == ";":
                    j += 1
                out.append("co_await std::suspend_always{};")
                i = j
                continue
            if t == "return" and self.barrier:
                out.append("co_return")
                i += 1
                continue
            # expression statement / control flow: translate up to the next ; { or }
            seg = []
            while i < n and toks[i] not in (";", "{", "}"):
                seg.append(toks[i])
                i += 1
            out.append(self._expr(seg, shadow))
            if i < n and toks[i] == ";":
                out.append(";")
                i += 1
        return "".join(out)

    def _expr(self, toks, shadow):
        shadowed = {s[0] for s in shadow}
        out = []
        i = 0
        n = len(toks)
        while i < n:
            t = toks[i]
            if t == "var":  # for-loop initialiser
                out.append("auto")
                i += 1
                continue
            if t == "bitcast":
                j = self._skip_ws(toks, i + 1)
                assert toks[j] == "<"
                ty, j = self._until(toks, j + 1, ">")
                out.append(f"bitcast_{self._type_text(ty)}")
                i = j + 1
                continue
            if t == "." and i + 1 < n and _SWIZZLE.match(toks[i + 1]):
                out.append("." + toks[i + 1] + "()")
                i += 2
                continue
            if t == "." and i + 1 < n:
                out.append("." + toks[i + 1])
                i += 2
                continue
            if t[0].isdigit() or (t[0] == "." and len(t) > 1):
                out.append(fix_number(t))
                i += 1
                continue
            if t in self.globals and t not in shadowed:
                out.append(f"G::{t}")
                i += 1
                continue
            out.append(t)
            i += 1
        return "".join(out)

    # -- top level --
    def translate(self):
        src = self.src
        src = src.replace("/*@UNIFORMS@*/", "").replace("/*@GRAPHUNIFORMS@*/", "")
        toks = tokenize(src)
        # pass 1: collect globals (bindings) so bodies can qualify them
        for m in re.finditer(r"@group\(\d+\)\s*@binding\((\d+)\)\s*var(?:<([^>]*)>)?\s+(\w+)\s*:\s*([^;]+);", src):
            idx, space, name, wtype = int(m.group(1)), (m.group(2) or "").replace(" ", ""), m.group(3), m.group(4)
            ctype = self._ctype(wtype)
            kind = "uniform" if space == "uniform" else ("storage" if space.startswith("storage") else "texture")
            if kind == "storage" and not ctype.startswith(("Storage", "AtomicU32")):
                ctype = f"Ref<{ctype}>"
            self.bindings.append((idx, kind, name, ctype))
            self.globals.add(name)

        decls = []
        funcs = []
        i = 0
        n = len(toks)
        pending_attrs = []
        while i < n:
            t = toks[i]
            if is_ws(t) or t == ";":
                i += 1
                continue
            if t == "@":
                j = self._skip_ws(toks, i + 1)
                attr = toks[j]
                j += 1
                args = None
                if j < n and toks[j] == "(":
                    a, j = self._until(toks, j + 1, ")")
                    args = "".join(a)
                    j += 1
                pending_attrs.append((attr, args))
                i = j
                continue
            if t == "override":
                j = self._skip_ws(toks, i + 1)
                name = toks[j]
                _, j = self._until(toks, j, ";")
                decls.append(f"constexpr u32 {name} = {self.overrides[name]}u;")
                i = j + 1
                pending_attrs = []
                continue
            if t == "const":
                j = self._skip_ws(toks, i + 1)
                name = toks[j]
                j = self._skip_ws(toks, j + 1)
                assert toks[j] == "="
                init, j = self._until(toks, j + 1, ";")
                decls.append(f"constexpr auto {name} ={self._expr(init, [])};")
                i = j + 1
                continue
            if t == "var":
                j = self._skip_ws(toks, i + 1)
                space = ""
                if toks[j] == "<":
                    sp, j = self._until(toks, j + 1, ">")
                    space = "".join(sp).replace(" ", "")
                    j = self._skip_ws(toks, j + 1)
                name = toks[j]
                ty, j = self._until(toks, self._skip_ws(toks, j + 1), ";")
                wtype = self._type_text(ty[1:] if ty and ty[0] == ":" else ty).lstrip(":")
                i = j + 1
                pending_attrs = []
                if space == "workgroup":
                    m = re.fullmatch(r"array<(\w+),(.+)>", wtype)
                    elem, size = _CTYPE[m.group(1)], m.group(2)
                    self.workgroup_vars.append((name, elem, size))
                    decls.append(f"static thread_local {elem} {name}[{self._expr(tokenize(size), [])}];")
                continue  # bindings were collected in pass 1
            if t == "fn":
                j = self._skip_ws(toks, i + 1)
                fname = toks[j]
                j = self._skip_ws(toks, j + 1)
                assert toks[j] == "("
                ptoks, j = self._until(toks, j + 1, ")")
                j = self._skip_ws(toks, j + 1)
                ret = "void"
                if toks[j] == "->":
                    rt, j = self._until(toks, self._skip_ws(toks, j + 1), "{")
                    ret = self._ctype(self._type_text(rt))
                assert toks[j] == "{"
                body, j = self._until(toks, j + 1, "}")
                i = j + 1
                attrs = dict(pending_attrs)
                pending_attrs = []
                # parameters
                params = []
                for p in "".join(ptoks).split(","):
                    p = p.strip()
                    if not p:
                        continue
                    bm = re.match(r"@builtin\((\w+)\)\s*(\w+)\s*:\s*(\w+)", p)
                    if bm:
                        self.builtins.append(bm.group(1))
                        params.append(f"{_CTYPE[bm.group(3)]} {bm.group(2)}")
                    else:
                        pn, pt = [x.strip() for x in p.split(":", 1)]
                        params.append(f"{self._ctype(pt)} {pn}")
                body_c = self._body(body)
                if "compute" in attrs:
                    ws = [x.strip() for x in attrs["workgroup_size"].split(",")]
                    while len(ws) < 3:
                        ws.append("1")
                    self.wgsize = ws
                    rtype = "Task" if self.barrier else "void"
                    funcs.append(f"{rtype} shader_main({', '.join(params)}) {{{body_c}}}")
                else:
                    funcs.append(f"{ret} {fname}({', '.join(params)}) {{{body_c}}}")
                continue
            raise ValueError(f"{self.name}: unexpected top-level token {t!r}")

        ns = self.name
        lines = ['#include "wgsl_rt.h"', '#include "uniforms_gen.h"', f"namespace {ns} {{", "using namespace wgsl;"]
        lines.append("namespace G {")
        for idx, kind, name, ctype in sorted(self.bindings):
            lines.append(f"{ctype} {name}{{}};")
        lines.append("}")
        lines += decls
        lines += funcs
        # entry wrapper: builtins in main's declared order
        names = {"global_invocation_id": "gid", "local_invocation_id": "lid",
                 "num_workgroups": "nwg", "workgroup_id": "wid"}
        args = ", ".join(names[b] for b in self.builtins)
        rtype = "Task" if self.barrier else "void"
        lines.append(f"{rtype} entry(vec3u gid, vec3u lid, vec3u nwg, vec3u wid) {{ (void)gid; (void)lid; (void)nwg; (void)wid; return shader_main({args}); }}")
        zero = " ".join(f"std::memset({w}, 0, sizeof({w}));" for w, _, _ in self.workgroup_vars)
        lines.append(f"void reset_wg() {{ {zero} }}")
        lines.append("}  // namespace " + ns)
        # C ABI: bind + dispatch
        lines.append(f'extern "C" void {ns}_bind(int b, void* p) {{')
        lines.append("  using namespace wgsl;")
        lines.append("  switch (b) {")
        for idx, kind, name, ctype in sorted(self.bindings):
            q = f"{ns}::G::{name}"
            if kind == "uniform":
                lines.append(f"  case {idx}: std::memcpy(&{q}, p, sizeof({q})); break;")
            elif ctype in ("TexF", "TexI", "TexW"):
                lines.append(f"  case {idx}: {q}.t = (TexData*)p; break;")
            elif ctype == "AtomicU32":
                lines.append(f"  case {idx}: {q}.p = (u32*)p; break;")
            else:
                lines.append(f"  case {idx}: {q}.p = (decltype({q}.p))p; break;")
        lines.append("  default: break;")
        lines.append("  }")
        lines.append("}")
        wx, wy, wz = [f"(unsigned)({ns}::{w})" if not w.isdigit() else w for w in self.wgsize]
        lines.append(f'extern "C" void {ns}_dispatch(unsigned nx, unsigned ny, unsigned nz) {{')
        if self.barrier:
            lines.append(f"  wgsl::run_barrier(&{ns}::entry, &{ns}::reset_wg, {wx}, {wy}, {wz}, nx, ny, nz);")
        else:
            lines.append(f"  wgsl::run_plain(&{ns}::entry, {wx}, {wy}, {wz}, nx, ny, nz);")
        lines.append("}")
        lines.append(f'extern "C" void {ns}_wgsize(unsigned* w) {{ w[0] = {wx}; w[1] = {wy}; w[2] = {wz}; }}')
        return "\n".join(lines) + "\n"


# Shader modules of the compute path (render shaders need a graphics API and are left out).
MODULES = {
    "ausm.js": [
        "prepareStateShaderCode", "boundaryShaderCode",
        "SLAU2_verticalFluxShaderCode", "SLAU2_horizontalFluxShaderCode",
        "SLAU_verticalFluxShaderCode", "SLAU_horizontalFluxShaderCode",
        "AUSMup_verticalFluxShaderCode", "AUSMup_horizontalFluxShaderCode",
        "residualShaderCode", "integrationStage1ShaderCode", "integrationStage2ShaderCode",
        "integrationStage3ShaderCode", "cflReductionShaderCode", "visualizationShaderCode",
    ],
    "grid.js": ["gridInterpolationShaderCode", "gridEllipticPoissonShaderCode", "gridFinalizeShaderCode"],
    "graphs.js": ["forceCalcShaderCode", "forceIntegrationShaderCode"],
}


# Field probe: the reference's visualization shader with its final colour-mapped store
# replaced by a store of the raw field value of the display mode (density, temperature,
# pressure, Mach, entropy) into the shader's own f32 buffer (binding 5), so that the
# headless field outputs can be compared with the reference's own arithmetic.  One
# statement is rewritten; everything before it is the reference's text.
PROBE_SRC = "visualizationShaderCode"
PROBE_NAME = "visualizationFieldProbe"
PROBE_FROM = ("textureStore(vis, gid.xy, colorMapBRYW(((localValue - freeStreamValue) * uni.visMultiplier)"
              " / (freeStreamValue * 2) + 0.5));")
PROBE_TO = "waveSpeeds[gid.x + gid.y * u32(uni.simDomain.x)] = localValue;"


def probe_source(wgsl: str) -> str:
    if wgsl.count(PROBE_FROM) != 1:
        raise ValueError("field probe: the visualization shader's final store was not found exactly once")
    return wgsl.replace(PROBE_FROM, PROBE_TO)


def uniforms_header(uni_fields, guni_fields):
    out = ["#pragma once", '#include "wgsl_rt.h"', "namespace wgsl {"]
    for sname, fields in (("Uniforms", uni_fields), ("GraphUniforms", guni_fields)):
        out.append(f"struct {sname} {{")
        for fname, ftype in fields:
            out.append(f"  {_CTYPE[ftype]} {fname}{{}};")
        out.append("};")
    out.append("}  // namespace wgsl")
    return "\n".join(out) + "\n"


def translate_reference(ref_root: Path, out_dir: Path):
    src = ref_root / "src"
    util_js = (src / "util.js").read_text()
    main_js = (src / "main.js").read_text()
    uni_fields = uniform_fields(util_js, "uni")
    guni_fields = uniform_fields(util_js, "graphUni")
    overrides = workgroup_overrides(main_js)
    out_dir.mkdir(parents=True, exist_ok=True)
    (out_dir / "uniforms_gen.h").write_text(uniforms_header(uni_fields, guni_fields))
    tpl = Templates()
    for fname in MODULES:
        tpl.load(src / "shaders" / fname)
    written = []
    for fname, names in MODULES.items():
        for name in names:
            wgsl = tpl.expand(name)
            mod = Module(name, wgsl, overrides, uni_fields, guni_fields)
            cpp = mod.translate()
            p = out_dir / f"{name}.cpp"
            p.write_text(cpp)
            written.append(p)
    wgsl = probe_source(tpl.expand(PROBE_SRC))
    p = out_dir / f"{PROBE_NAME}.cpp"
    p.write_text(Module(PROBE_NAME, wgsl, overrides, uni_fields, guni_fields).translate())
    written.append(p)
    return written


if __name__ == "__main__":
    if len(sys.argv) < 2:
        sys.exit("usage: translate.py REFERENCE_ROOT [OUT_DIR]")
    ref = Path(sys.argv[1])
    out = Path(sys.argv[2]) if len(sys.argv) > 2 else Path(__file__).resolve().parents[1] / "_ref" / "gen"
    for p in translate_reference(ref, out):
        print(p)
