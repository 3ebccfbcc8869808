"""Reader and writer of KAPSEL's UDF files (the OCTA "user definable format").

The reference reads its input through OCTA's UDFManager (Gourmet_file_io,
input.cxx:438-1818) and writes output and restart records through it
(Output_udf avs_output.cxx:343-450, Save_Restart_udf resume.cxx:10-78).  A
UDF file has definition blocks (``\\begin{def}`` / ``\\begin{global_def}``,
possibly pulled in by ``\\include{"define.udf"}``) that declare classes and
named entries with types, and a ``\\begin{data}`` block whose values are
positional: a struct is ``{v1, v2, ...}`` in declaration order, an array is
``[e0, e1, ...]``, a ``select`` is a string, and braces of consecutive
structs may abut (``}{``).

This module parses both parts, pairs each value with its declared type and
flattens the result into the dotted paths the reference asks for (for
example ``constitutive_eq.Navier_Stokes.DX`` or
``object_type.spherical_particle.Particle_spec[0].Particle_number``).
``write`` serialises such a structure back in the positional form, and
``to_config`` turns a flattened input file into the configuration dict of
``kapsel_old_b200.Simulation``.
"""
from __future__ import annotations

import math
import os
import re

__all__ = ["parse", "read", "flatten", "write", "write_records", "read_records", "to_config", "UDFError"]


class UDFError(ValueError):
    pass


_TOK = re.compile(r"""
    (?P<ws>\s+)
  | (?P<comment>//[^\n]*)
  | (?P<cmd>\\[A-Za-z_]+\{[^}]*\})
  | (?P<str>"(?:[^"\\]|\\[\s\S])*"|'(?:[^'\\]|\\[\s\S])*')
  | (?P<num>[-+]?(?:\d+\.?\d*|\.\d+)(?:[eE][-+]?\d+)?(?![A-Za-z_]))
  | (?P<name>[A-Za-z_][A-Za-z0-9_]*)
  | (?P<punct>[{}\[\],:;])
""", re.X)


def _tokens(text: str):
    out = []
    pos = 0
    while pos < len(text):
        m = _TOK.match(text, pos)
        if not m:
            raise UDFError(f"unexpected character {text[pos]!r} at offset {pos}")
        pos = m.end()
        kind = m.lastgroup
        if kind in ("ws", "comment"):
            continue
        out.append((kind, m.group(kind)))
    return out


# ---------------------------------------------------------------------------
# types
class _T:
    """A declared type: kind in {'scalar', 'select', 'struct', 'class'}."""

    def __init__(self, kind, base=None, fields=None, choices=None, name=None):
        self.kind, self.base, self.fields, self.choices, self.name = kind, base, fields, choices, name

    def __repr__(self):
        return f"_T({self.kind}, {self.base or self.name or ''})"


class _Field:
    def __init__(self, name, dims, typ):
        self.name, self.dims, self.typ = name, dims, typ


class _Reader:
    def __init__(self, toks):
        self.t, self.i = toks, 0

    def peek(self, k=0):
        return self.t[self.i + k] if self.i + k < len(self.t) else (None, None)

    def next(self):
        tok = self.peek()
        self.i += 1
        return tok

    def expect(self, val):
        kind, v = self.next()
        if v != val:
            raise UDFError(f"expected {val!r}, found {v!r}")

    def accept(self, val):
        if self.peek()[1] == val:
            self.i += 1
            return True
        return False


_SCALARS = {"double", "float", "int", "string"}


def _parse_type(r: _Reader, classes):
    kind, v = r.next()
    if v == "{":
        fields = _parse_fields(r, classes, "}")
        t = _T("struct", fields=fields)
    elif v == "select":
        r.expect("{")
        choices = []
        while not r.accept("}"):
            k, s = r.next()
            if k == "str":
                choices.append(s[1:-1])
            elif s != ",":
                raise UDFError(f"bad select entry {s!r}")
        t = _T("select", choices=choices)
    elif v in _SCALARS:
        t = _T("scalar", base=v)
    elif kind == "name":
        if v not in classes:
            raise UDFError(f"unknown type {v!r}")
        t = classes[v]
    else:
        raise UDFError(f"bad type token {v!r}")
    while r.peek()[0] == "str":  # descriptions after a type
        r.next()
    return t


def _parse_fields(r: _Reader, classes, close):
    fields = []
    while not r.accept(close):
        if r.accept(","):
            continue
        kind, name = r.next()
        if kind != "name":
            raise UDFError(f"expected a field name, found {name!r}")
        dims = 0
        while r.accept("["):
            r.expect("]")
            dims += 1
        r.expect(":")
        fields.append(_Field(name, dims, _parse_type(r, classes)))
    return fields


class _Defs:
    def __init__(self):
        self.classes = {}
        self.entries = []  # top-level _Field list in declaration order

    def add_block(self, toks):
        r = _Reader(toks)
        while r.peek()[0] is not None:
            if r.accept(",") or r.accept(";"):
                continue
            kind, v = r.peek()
            if v == "class":
                r.next()
                _, name = r.next()
                r.expect(":")
                t = _parse_type(r, self.classes)
                self.classes[name] = t
            else:
                self.entries.extend(_parse_fields_one(r, self.classes))

    def entry(self, name):
        for f in self.entries:
            if f.name == name:
                return f
        raise UDFError(f"no definition for {name!r}")


def _parse_fields_one(r: _Reader, classes):
    kind, name = r.next()
    if kind != "name":
        raise UDFError(f"expected a definition name, found {name!r}")
    dims = 0
    while r.accept("["):
        r.expect("]")
        dims += 1
    r.expect(":")
    return [_Field(name, dims, _parse_type(r, classes))]


# ---------------------------------------------------------------------------
# values
def _scalar(tok, typ):
    kind, v = tok
    if kind == "str":
        return v[1:-1]
    if kind == "num":
        if typ.kind == "scalar" and typ.base == "int":
            return int(float(v))
        return float(v)
    if kind == "name":  # bare words (rare)
        return v
    raise UDFError(f"expected a value, found {v!r}")


def _parse_value(r: _Reader, typ, dims):
    if dims > 0:
        r.expect("[")
        out = []
        while not r.accept("]"):
            if r.accept(","):
                continue
            out.append(_parse_value(r, typ, dims - 1))
        return out
    if typ.kind == "struct":
        r.expect("{")
        out = {}
        for f in typ.fields:
            while r.accept(","):
                pass
            out[f.name] = _parse_value(r, f.typ, f.dims)
        while r.accept(","):
            pass
        r.expect("}")
        return out
    return _scalar(r.next(), typ)


def _blocks(text: str):
    """(name, body) of every \\begin{name} ... \\end{name} block at top level,
    and the \\include file names, in order."""
    out = []
    pat = re.compile(r"\\(begin|end|include)\{([^}]*)\}")
    depth, start, name = 0, 0, None
    for m in pat.finditer(text):
        kind, arg = m.group(1), m.group(2)
        if kind == "include" and depth == 0:
            out.append(("include", arg.strip().strip('"')))
        elif kind == "begin":
            if depth == 0:
                name, start = arg, m.end()
            depth += 1
        elif kind == "end":
            depth -= 1
            if depth == 0:
                out.append((name, text[start:m.start()]))
    return out


def parse(text: str, base_dir: str = ".", defs: _Defs | None = None):
    """(definitions, data) of UDF text; data maps entry names to values."""
    defs = defs or _Defs()
    data = {}
    for name, body in _blocks(text):
        if name == "include":
            path = body if os.path.isabs(body) else os.path.join(base_dir, body)
            with open(path) as f:
                parse(f.read(), os.path.dirname(path), defs)
        elif name in ("def", "global_def"):
            defs.add_block(_tokens(body))
        elif name == "data":
            r = _Reader(_tokens(body))
            while r.peek()[0] is not None:
                if r.accept(",") or r.accept(";"):
                    continue
                kind, ent = r.next()
                dims = 0
                while r.accept("["):
                    r.expect("]")
                    dims += 1
                r.expect(":")
                f = defs.entry(ent)
                data[ent] = _parse_value(r, f.typ, f.dims)
        # the header block and others carry no simulation data
    return defs, data


def read(path: str):
    """Flattened `path -> value` map of a UDF file (includes resolved)."""
    with open(path) as f:
        defs, data = parse(f.read(), os.path.dirname(os.path.abspath(path)))
    return flatten(data)


def flatten(data: dict, prefix: str = "") -> dict:
    out = {}

    def rec(v, p):
        if isinstance(v, dict):
            for k, x in v.items():
                rec(x, f"{p}.{k}" if p else k)
        elif isinstance(v, list):
            for i, x in enumerate(v):
                rec(x, f"{p}[{i}]")
        else:
            out[p] = v

    rec(data, prefix)
    return out


# ---------------------------------------------------------------------------
def _fmt(v, typ):
    if isinstance(v, str):
        return '"' + v + '"'
    if typ.kind == "scalar" and typ.base == "int":
        return str(int(v))
    return repr(float(v))


def _write_value(v, typ, dims, ind):
    pad = " " * ind
    if dims > 0:
        if not v:
            return "[]"
        return "[" + ",".join(_write_value(x, typ, dims - 1, ind + 1) for x in v) + "]"
    if typ.kind == "struct":
        parts = [_write_value(v[f.name], f.typ, f.dims, ind + 1) for f in typ.fields]
        return "{" + ",".join(parts) + "}"
    return _fmt(v, typ)


def write(path: str, data: dict, define_file: str, defs: _Defs | None = None):
    """Write `data` (entry name -> nested value) as a UDF data block that
    includes `define_file`, in the declaration order of the definitions."""
    if defs is None:
        with open(define_file if os.path.isabs(define_file) else
                  os.path.join(os.path.dirname(os.path.abspath(path)), define_file)) as f:
            defs, _ = parse(f.read(), os.path.dirname(os.path.abspath(path)))
    lines = [f'\\include{{"{os.path.basename(define_file)}"}}', "", "\\begin{data}"]
    for fdef in defs.entries:
        if fdef.name in data:
            lines.append(f"{fdef.name}:{_write_value(data[fdef.name], fdef.typ, fdef.dims, 1)}")
    lines.append("\\end{data}")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def write_records(path: str, records: list, define_file: str, header: dict | None = None,
                  defs: _Defs | None = None):
    """Write an output UDF: the definitions by ``\\include``, then one
    ``\\begin{data}`` block per record, values positional in declaration
    order.  `header` (entry name -> nested value), when given, is record 0:
    the input values the reference echoes into its output file before the
    first snapshot (Gourmet_file_io); each later record is one Output_udf
    call (avs_output.cxx:343-450: E, t, Particles[])."""
    if defs is None:
        with open(define_file if os.path.isabs(define_file) else
                  os.path.join(os.path.dirname(os.path.abspath(path)), define_file)) as f:
            defs, _ = parse(f.read(), os.path.dirname(os.path.abspath(path)))
    lines = [f'\\include{{"{os.path.basename(define_file)}"}}', ""]
    for rec in ([header] if header else []) + list(records):
        lines.append("\\begin{data}")
        for fdef in defs.entries:
            if fdef.name in rec:
                lines.append(f"{fdef.name}:{_write_value(rec[fdef.name], fdef.typ, fdef.dims, 1)}")
        lines.append("\\end{data}")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def read_records(path: str) -> list:
    """Flattened `path -> value` map of every ``\\begin{data}`` block of a
    UDF file, in order (one per record)."""
    with open(path) as f:
        text = f.read()
    base = os.path.dirname(os.path.abspath(path))
    defs = _Defs()
    out = []
    for name, body in _blocks(text):
        if name == "include":
            p = body if os.path.isabs(body) else os.path.join(base, body)
            with open(p) as g:
                parse(g.read(), os.path.dirname(p), defs)
        elif name in ("def", "global_def"):
            defs.add_block(_tokens(body))
        elif name == "data":
            _, data = parse("\\begin{data}" + body + "\\end{data}", base, defs)
            out.append(flatten(data))
    return out


# ---------------------------------------------------------------------------
def _on(v) -> bool:
    return str(v) == "ON"


def to_config(flat: dict, seed: int = 0) -> dict:
    """Configuration dict of `Simulation` from a flattened input UDF (one
    spherical-particle species, Navier_Stokes or Electrolyte), following
    Gourmet_file_io (input.cxx:438-1818) and the automatic time step of
    Set_global_parameters (input.cxx:316-362: DT = factor / (NU KMAX2), the
    Electrolyte taking the smaller of that and the ion diffusion time).
    Particles placed by the reference's unseeded rand() (uniform_random,
    random_walk, FCC, BCC) are placed here by the seeded non-overlapping
    sampler instead; user_specify positions and orientations are kept."""
    g = flat.get
    eq = g("constitutive_eq.type")
    if eq not in ("Navier_Stokes", "Electrolyte"):
        raise UDFError(f"constitutive_eq {eq!r} is not supported")
    b = f"constitutive_eq.{eq}."
    if g("object_type.type") != "spherical_particle":
        raise UDFError("only object_type spherical_particle is supported")
    nspec = sum(1 for k in flat if re.fullmatch(r"object_type\.spherical_particle\.Particle_spec\[\d+\]\.Particle_number", k))
    if nspec != 1:
        raise UDFError("exactly one particle species is supported")
    ps = "object_type.spherical_particle.Particle_spec[0]."
    if g(ps + "janus_propulsion", "OFF") != "OFF":
        raise UDFError("self-propelled (janus) particles are not supported")
    npx = [int(g(f"mesh.NP{c}")) for c in "XYZ"]
    cfg = {
        "eq": eq,
        "np_xyz": tuple(npx),
        "dx": float(g(b + "DX")), "rho": float(g(b + "RHO")), "eta": float(g(b + "ETA")),
        "kbt": float(g(b + "kBT")), "alpha_v": float(g(b + "alpha_v")), "alpha_o": float(g(b + "alpha_o")),
        "a": float(g("A")), "a_xi": float(g("A_XI")),
        "mass_ratio": float(g(ps + "MASS_RATIO")),
        "gravity_g": float(g("gravity.G", 0.0)), "gravity_dir": g("gravity.G_direction", "-Z"),
        "epsilon": float(g("EPSILON")), "lj_powers": g("LJ_powers"),
        "rotation": g("switch.ROTATION", "ON"), "lj_truncate": g("switch.LJ_truncate", "ON"),
        "fix_cell": tuple(_on(g(f"switch.FIX_CELL.{c}", "OFF")) for c in "xyz"),
        "output": {"GTS": int(g("output.GTS", 1)), "Num_snap": int(g("output.Num_snap", 0))},
    }
    # time step
    if g("time_increment.type") == "manual":
        cfg["dt"] = float(g("time_increment.manual.delta_t"))
    else:
        nu = cfg["eta"] / cfg["rho"]
        n = [1 << p for p in npx]
        kmax2 = sum((2.0 * math.pi / (n[d] * cfg["dx"]) * ((n[d] + 2) // 3)) ** 2 for d in range(3))
        tdump = 1.0 / (nu * kmax2)
        if eq == "Electrolyte":
            salt = g(b + "Add_salt.type") == "salt"
            ons = (max(float(g(b + "Add_salt.salt.Onsager_coeff_positive_ion")),
                       float(g(b + "Add_salt.salt.Onsager_coeff_negative_ion"))) if salt else
                   float(g(b + "Add_salt.saltfree.Onsager_coeff_counterion")))
            tdump = min(tdump, 1.0 / (cfg["kbt"] * ons * kmax2))
        cfg["dt"] = float(g("time_increment.auto.factor")) * tdump
    # particles
    nparts = int(g(ps + "Particle_number"))
    init = g("switch.INIT_distribution.type")
    if init == "user_specify":
        up = "switch.INIT_distribution.user_specify.Particles"
        parts = []
        for i in range(nparts):
            p = f"{up}[{i}]."
            x = tuple(float(g(p + f"R.{c}")) for c in "xyz")
            q = tuple(float(g(p + f"q.q{j}", 1.0 if j == 0 else 0.0)) for j in range(4))
            parts.append({"x": x, "q": q})
        cfg["particles"] = parts
    else:
        from .workload import place_spheres

        n = [(1 << p) * cfg["dx"] for p in npx]
        xs = place_spheres(nparts, n, cfg["a"] * cfg["dx"], 0.05 * cfg["a"] * cfg["dx"], seed)
        cfg["particles"] = [{"x": tuple(float(c) for c in x)} for x in xs]
    if eq == "Electrolyte":
        if g(b + "Add_salt.type") != "salt" or g(b + "INIT_profile") != "Uniform":
            raise UDFError("only the salt case with a Uniform initial profile is supported")
        s = b + "Add_salt.salt."
        ef = (0.0, 0.0, 0.0)
        if g(b + "Electric_field.type") == "ON":
            if g(b + "Electric_field.ON.type") != "DC":
                raise UDFError("only a DC external field is supported")
            ef = tuple(float(g(b + f"Electric_field.ON.DC.E{c}")) for c in "xyz")
        cfg["electrolyte"] = {
            "dielectric": float(g(b + "Dielectric_cst")), "surface_charge": float(g(ps + "Surface_charge")),
            "debye": float(g(s + "Debye_length")), "val_p": float(g(s + "Valency_positive_ion")),
            "val_n": float(g(s + "Valency_negative_ion")), "onsager_p": float(g(s + "Onsager_coeff_positive_ion")),
            "onsager_n": float(g(s + "Onsager_coeff_negative_ion")), "efield": ef}
        cfg["alpha_v"] = cfg["alpha_v"]
    return cfg
