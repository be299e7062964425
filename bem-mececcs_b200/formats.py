"""Input and output file formats of BEM-MECECCS.

The static input (read by INPUTECE, src/Inputece.for:16-108) and its echo in
the static output, the dynamic input (INPUTECD, src/Inputecd.for:7-139) and
the per-frequency result block of the dynamic output (OUTPUTEC,
src/Outputec.for:9-68).  Files are Latin-1 text; numbers are read with
Fortran list-directed semantics: every READ statement starts on a new
record, takes as many values as it needs across records and drops the rest
of its last record.
"""
from __future__ import annotations

import dataclasses
import re

import numpy as np

_ENC = "latin-1"


@dataclasses.dataclass
class StaticInput:
    """Everything INPUTECE reads (src/Inputece.for:35-102)."""

    title: str
    n: int          # elements in the mesh (boundary + enclosing)
    nbe: int        # boundary elements (collocation points)
    np: int         # nodes
    npg: int        # Gauss points per direction
    ge: float       # shear modulus
    rnu: float      # Poisson ratio
    cx: np.ndarray  # (np,) node coordinates
    cy: np.ndarray
    cz: np.ndarray
    cone: np.ndarray  # (n, 4) int32, 1-based node numbers

    def cone_fortran(self) -> np.ndarray:
        """CONE(N,4) in Fortran column-major order, as the C-ABI expects."""
        return np.asfortranarray(self.cone.astype(np.int32)).ravel(order="F")

    def centroids(self):
        """CXM/CYM/CZM, src/Inputece.for:100-102."""
        c = self.cone - 1
        return tuple((a[c[:, 0]] + a[c[:, 1]] + a[c[:, 2]] + a[c[:, 3]]) * 0.250
                     for a in (self.cx, self.cy, self.cz))


@dataclasses.dataclass
class DynamicInput:
    """Everything INPUTECD reads (src/Inputecd.for:30-134)."""

    title: str
    l: int            # interior points
    nfr: int          # frequencies
    dam: float        # hysteretic damping
    rho: float        # density
    freqs: np.ndarray  # (nfr,)
    kode: np.ndarray  # (3*nbe,) int32: 0 displacement prescribed, 1 traction
    bc: np.ndarray    # (3*nbe,) prescribed values
    cxi: np.ndarray   # (l,) interior points
    cyi: np.ndarray
    czi: np.ndarray


class _Records:
    """Fortran list-directed reader over the lines of a file."""

    _split = re.compile(r"[\s,]+")

    def __init__(self, lines):
        self.lines = lines
        self.pos = 0

    def line(self) -> str:
        s = self.lines[self.pos]
        self.pos += 1
        return s

    def read(self, count: int) -> list:
        vals: list = []
        while len(vals) < count:
            if self.pos >= len(self.lines):
                raise EOFError("list-directed read ran past the end of file")
            toks = [t for t in self._split.split(self.lines[self.pos].strip()) if t]
            self.pos += 1
            vals.extend(toks)
        return vals[:count]


def _f(tok: str) -> float:
    return float(tok.replace("D", "E").replace("d", "e"))


def read_static(path) -> StaticInput:
    with open(path, encoding=_ENC) as fh:
        rec = _Records(fh.read().splitlines())
    title = rec.line()
    n, nbe, np_, npg, ge, rnu = rec.read(6)
    n, nbe, np_, npg = int(n), int(nbe), int(np_), int(npg)
    xyz = np.array([_f(t) for t in rec.read(3 * np_)]).reshape(np_, 3)
    cone = np.zeros((n, 4), dtype=np.int32)
    for i in range(n):  # READ(INP,*) (cone_in(J),J=1,4); CONE = INT(cone_in)
        cone[i] = [int(_f(t)) for t in rec.read(4)]
    return StaticInput(title, n, nbe, np_, npg, _f(ge), _f(rnu),
                       xyz[:, 0].copy(), xyz[:, 1].copy(), xyz[:, 2].copy(), cone)


def read_dynamic(path, nbe: int) -> DynamicInput:
    with open(path, encoding=_ENC) as fh:
        rec = _Records(fh.read().splitlines())
    title = rec.line()
    l, nfr, dam, rho = rec.read(4)
    l, nfr = int(l), int(nfr)
    freqs = np.array([_f(t) for t in rec.read(nfr)])
    kode = np.zeros(3 * nbe, dtype=np.int32)
    bc = np.zeros(3 * nbe)
    for i in range(nbe):  # READ(INQ,*) (KODE(3*(I-1)+J),BC(3*(I-1)+J),J=1,3)
        t = rec.read(6)
        for j in range(3):
            kode[3 * i + j] = int(_f(t[2 * j]))
            bc[3 * i + j] = _f(t[2 * j + 1])
    if l > 0:
        p = np.array([_f(t) for t in rec.read(3 * l)]).reshape(l, 3)
    else:
        p = np.zeros((0, 3))
    return DynamicInput(title, l, nfr, _f(dam), _f(rho), freqs, kode, bc,
                        p[:, 0].copy(), p[:, 1].copy(), p[:, 2].copy())


def _fmt_i(v, width: int) -> str:
    """Fortran Iw: right-justified, or `width` asterisks when the number does
    not fit."""
    t = str(int(v))
    return t.rjust(width) if len(t) <= width else "*" * width


def _r(v) -> str:
    """Shortest decimal that reads back to the same double."""
    return repr(float(v))


def write_static(path, s: StaticInput) -> None:
    """Writes a file INPUTECE reads back unchanged."""
    out = [s.title, " ", f"{s.n} {s.nbe} {s.np} {s.npg} {_r(s.ge)} {_r(s.rnu)}", ""]
    out += [f" {_r(x)} {_r(y)} {_r(z)}" for x, y, z in zip(s.cx, s.cy, s.cz)]
    out += [" " + " ".join(f"{int(v)}." for v in row) for row in s.cone]
    with open(path, "w", encoding=_ENC) as fh:
        fh.write("\n".join(out) + "\n")


def format_static_echo(s: StaticInput) -> str:
    """The static output file: INPUTECE's echo of what it read, with the
    element centroids it computes (src/Inputece.for:29-104; formats 100, 200,
    300, 400, 500, 550).  The reference's known-answer test requires this file
    to equal the shipped SSOLO*E_-5+5.SOL byte for byte (src/tests.sh:43)."""
    def d(v, w, k):
        return _fmt_d(float(v), w, k)

    out = ["", " " + "*" * 79, "", f"{s.title[:75]:<75s}", "", "", "DADOS", "",
           f"  N\xdaMERO DE ELEMENTOS DA MALHA= {_fmt_i(s.n, 4)}",
           f"  N\xdaMERO DE ELEMENTOS DE CONTORNO= {_fmt_i(s.nbe, 4)}",
           f"  N\xdaMERO DE PONTOS EXTREMOS DOS ELEMENTOS= {_fmt_i(s.np, 4)}",
           f"  N\xdaMERO DE PONTOS DE GAUSS= {_fmt_i(s.npg, 3)}",
           f"  M\xd3DULO DE CISALHAMENTO= {d(s.ge, 14, 7)}",
           f"  COEFICIENTE DE POISSON= {d(s.rnu, 14, 7)}",
           "", "", "  COORDENADAS DOS PONTOS EXTREMOS DOS ELEMENTOS DE CONTORNO", "",
           f"    PONTO{'':10s}X{'':18s}Y{'':18s}Z"]
    out += [f"    {_fmt_i(i + 1, 4)}" + "".join(f"     {d(v, 14, 7)}" for v in xyz)
            for i, xyz in enumerate(zip(s.cx, s.cy, s.cz))]
    out += ["", "", "  CONECTIVIDADE DOS ELEMENTOS DE CONTORNO", "",
            f" ELEMENTO{'':3s}EXTR I{'':3s}EXTR J{'':3s}EXTR K{'':3s}EXTR L"
            f"{'':5s}XMED{'':8s}YMED{'':8s}ZMED"]
    cxm, cym, czm = s.centroids()
    out += [_fmt_i(i + 1, 6) + "".join(_fmt_i(c, 9) for c in s.cone[i]) + "  "
            + "".join(d(v, 12, 4) for v in (cxm[i], cym[i], czm[i]))
            for i in range(s.n)]
    return "\n".join(out) + "\n"


def format_dynamic_echo(s: StaticInput, d: DynamicInput, material) -> str:
    """The head of the dynamic output file: INPUTECD's echo of the mesh and of
    what it read, with the derived complex material `material` = (ZGE, ZCS,
    ZCP) (src/Inputecd.for:23-136; formats 100, 200, 230, 250, 300, 400, 500,
    550, 600, 650, 700, 750).  The result blocks of format_results follow it."""
    def f(v, w, k):
        return _fmt_d(float(v), w, k)

    zge, zcs, zcp = material
    out = ["", " " + "*" * 79, "", f"{d.title[:75]:<75s}", "", "", "DADOS", "",
           f"  N\xdaMERO DE ELEMENTOS DA MALHA= {_fmt_i(s.n, 4)}",
           f"  N\xdaMERO DE ELEMENTOS DE CONTORNO= {_fmt_i(s.nbe, 4)}",
           f"  N\xdaMERO DE PONTOS EXTREMOS DOS ELEMENTOS= {_fmt_i(s.np, 4)}",
           f"  N\xdaMERO DE PONTOS INTERNOS= {_fmt_i(d.l, 3)}",
           f"  N\xdaMERO DE PONTOS DE GAUSS= {_fmt_i(s.npg, 3)}",
           f"  N\xdaMERO DE FREQ\xdc\xcaNCIAS= {_fmt_i(d.nfr, 3)}",
           f"  M\xd3DULO DE CISALHAMENTO (REAL)= {f(s.ge, 14, 7)}",
           f"  COEFICIENTE DE POISSON= {f(s.rnu, 14, 7)}",
           f"  COEFICIENTE DE AMORTECIMENTO= {f(d.dam, 14, 7)}",
           f"  DENSIDADE DE MASSA= {f(d.rho, 14, 7)}",
           "", "", "DADOS DERIVADOS", "",
           f"  M\xd3DULO DE CISALHAMENTO (COMPLEXO)= {f(zge.real, 14, 7)}{f(zge.imag, 14, 7)}",
           f"  VELOCIDADE DA ONDA-S (COMPLEXO)= {f(zcs.real, 14, 7)}{f(zcs.imag, 14, 7)}",
           f"  VELOCIDADE DA ONDA-P (COMPLEXO)= {f(zcp.real, 14, 7)}{f(zcp.imag, 14, 7)}",
           "", "  FREQUENCIAS", ""]
    fr = list(d.freqs)
    out += ["".join(f"  {f(v, 14, 7)}" for v in fr[k:k + 5]) for k in range(0, len(fr), 5)]
    out += ["", "", "  COORDENADAS DOS PONTOS EXTREMOS DOS ELEMENTOS DA MALHA", "",
            f"    PONTO{'':10s}X{'':18s}Y{'':18s}Z"]
    out += [f"    {_fmt_i(i + 1, 4)}" + "".join(f"     {f(v, 14, 7)}" for v in xyz)
            for i, xyz in enumerate(zip(s.cx, s.cy, s.cz))]
    out += ["", "", "  CONECTIVIDADE DOS ELEMENTOS DA MALHA", "",
            f" ELEMENTO{'':3s}EXTR I{'':3s}EXTR J{'':3s}EXTR K{'':3s}EXTR L"
            f"{'':5s}XMED{'':8s}YMED{'':8s}ZMED"]
    cxm, cym, czm = s.centroids()
    out += [_fmt_i(i + 1, 6) + "".join(_fmt_i(c, 9) for c in s.cone[i]) + "  "
            + "".join(f(v, 12, 4) for v in (cxm[i], cym[i], czm[i]))
            for i in range(s.n)]
    out += ["", "", "  CONDI\xc7\xd5ES DE CONTORNO", "",
            (f"{'':8s}" + f"VALOR PRESCRITO{'':10s}" * 3).rstrip(),  # a final nX writes nothing
            f" ELEM{'':6s}DIRE\xc7\xc3O X{'':4s}C\xd3DIGO{'':6s}DIRE\xc7\xc3O Y{'':4s}C\xd3DIGO"
            f"{'':6s}DIRE\xc7\xc3O Z{'':4s}C\xd3DIGO"]
    out += [(_fmt_i(i + 1, 4) + "".join(f"    {f(d.bc[3 * i + j], 10, 3)}      "
                                        f"{_fmt_i(d.kode[3 * i + j], 3)}  " for j in range(3))).rstrip()
            for i in range(s.nbe)]
    if d.l > 0:
        out += ["", "", "  COORDENADAS DOS PONTOS INTERNOS ", "",
                f"    PONTO{'':10s}X{'':18s}Y{'':17s} Z"]
        out += [f"    {_fmt_i(i + 1, 3)}" + "".join(f(v, 19, 7) for v in xyz)
                for i, xyz in enumerate(zip(d.cxi, d.cyi, d.czi))]
    return "\n".join(out) + "\n"


def write_dynamic(path, d: DynamicInput) -> None:
    """Writes a file INPUTECD reads back unchanged."""
    out = [d.title, " ", f"{d.l} {d.nfr} {_r(d.dam)} {_r(d.rho)}", ""]
    out.append(" ".join(_r(f) for f in d.freqs))
    out.append("")
    nbe = len(d.kode) // 3
    for i in range(nbe):
        out.append("  ".join(f"{int(d.kode[3*i+j])} {_r(d.bc[3*i+j])}" for j in range(3)))
    out.append("")
    for x, y, z in zip(d.cxi, d.cyi, d.czi):
        out.append(f"{_r(x)} {_r(y)} {_r(z)}")
    with open(path, "w", encoding=_ENC) as fh:
        fh.write("\n".join(out) + "\n")


# --- OUTPUTEC result blocks (src/Outputec.for:21-59, format 200: D11.4 pairs)

_NUM = r"[-+]?\d*\.\d+[DE][-+]\d+"
_PAIR = re.compile(rf"({_NUM}),\s*({_NUM})")


def _pairs(line: str) -> list:
    return [complex(_f(a), _f(b)) for a, b in _PAIR.findall(line)]


@dataclasses.dataclass
class Results:
    """One frequency block of the dynamic output file."""

    freq: float
    disp: np.ndarray      # (nbe, 3) boundary displacements (ZFI after INTEREC)
    traction: np.ndarray  # (nbe, 3) boundary tractions (ZDFI after INTEREC)
    idisp: np.ndarray     # (l, 3) interior displacements (ZDSOL)
    sigma: np.ndarray     # (l, 9) interior stresses (ZSSOL)


def parse_results(path) -> list:
    """Parses every frequency block (Outputec.for:24-59) of an output file."""
    with open(path, encoding=_ENC) as fh:
        lines = fh.read().splitlines()
    blocks = []
    i = 0
    freq_re = re.compile(rf"=\s*({_NUM})")
    while i < len(lines):
        if "RESULTADOS" not in lines[i]:
            i += 1
            continue
        freq = np.nan
        for back in range(i - 1, max(i - 6, -1), -1):
            m = freq_re.search(lines[back])
            if m:
                freq = _f(m.group(1))
                break
        sections = {"disp": [], "traction": [], "idisp": [], "sigma": []}
        cur = None
        i += 1
        while i < len(lines) and "RESULTADOS" not in lines[i]:
            ln = lines[i]
            if "DESLOCAMENTO X" in ln and "ELEM" in ln:
                cur = "disp"
            elif "TRACTION X" in ln:
                cur = "traction"
            elif "DESLOCAMENTO X" in ln and "PONTO" in ln:
                cur = "idisp"
            elif "SIGMAXX" in ln:
                cur = "sigma"
            elif cur and re.match(r"^\s*\d+\s", ln):
                vals = _pairs(ln)
                if vals:
                    sections[cur].append(vals)
            i += 1
        blocks.append(Results(
            freq,
            np.array(sections["disp"], dtype=complex).reshape(-1, 3),
            np.array(sections["traction"], dtype=complex).reshape(-1, 3),
            np.array(sections["idisp"], dtype=complex).reshape(-1, 3),
            np.array(sections["sigma"], dtype=complex).reshape(-1, 9)))
    return blocks


def _fmt_d(v: float, width: int = 11, digits: int = 4) -> str:
    """Fortran Dw.d: 0.dddd D+ee with the leading zero kept (a three-digit
    exponent drops the D).  The digits are the correctly rounded decimal
    expansion of the double, taken from Python's %e conversion."""
    if v == 0.0:
        body = "0." + "0" * digits + "D+00"
    else:
        t = f"{abs(v):.{digits - 1}e}"  # d.ddde+XX, rounding carries included
        e = int(t[digits + 2:]) + 1
        mant = t[0] + t[2:digits + 1]
        body = (f"0.{mant}D{'+' if e >= 0 else '-'}{abs(e):02d}" if abs(e) < 100
                else f"0.{mant}{'+' if e >= 0 else '-'}{abs(e):03d}")
        if v < 0:
            body = "-" + body
    return body.rjust(width)


def format_results(r: Results) -> str:
    """The OUTPUTEC block (Outputec.for:21-59) for one frequency."""
    def row(idx, vals, w=5):
        return _fmt_i(idx, w) + "".join(f"  {_fmt_d(z.real)},{_fmt_d(z.imag)}" for z in vals)

    out = ["", " " + "*" * 79, "", f"{'':30s}FREQ\xdc\xcaNCIA = {_fmt_d(r.freq, 14, 7)}", "",
           " " + "*" * 79, "", " RESULTADOS", "", "  N\xd3S DO CONTORNO", "",
           " ELEM      DESLOCAMENTO X           DESLOCAMENTOT Y           DESLOCAMENTO Z", ""]
    out += [row(i + 1, v) for i, v in enumerate(r.disp)]
    out += ["", " ELEM        TRACTION X               TRACTION Y               TRACTION Z", ""]
    out += [row(i + 1, v) for i, v in enumerate(r.traction)]
    if len(r.idisp):
        out += ["", "", "  PONTOS INTERNOS", "",
                " PONTO     DESLOCAMENTO X           DESLOCAMENTO Y           DESLOCAMENTO Z"]
        out += [row(i + 1, v) for i, v in enumerate(r.idisp)]
        out += ["", "", "  PONTOS INTERNOS", "",
                " PONTO        SIGMAXX                 SIGMAXY                  SIGMAXZ"
                "                  SIGMAYX                  SIGMAYY                  SIGMAYZ"
                "                  SIGMAZX                  SIGMAZY                  SIGMAZZ"]
        out += [row(i + 1, v, 4) for i, v in enumerate(r.sigma)]
    out.append(" " + "*" * 230)
    return "\n".join(out) + "\n"


def write_dynamic_output(path, s: StaticInput, d: DynamicInput, material, results) -> None:
    """The dynamic output file the reference writes: INPUTECD's echo, then one
    OUTPUTEC block per frequency (`results`, a list of Results)."""
    with open(path, "w", encoding=_ENC) as fh:
        fh.write(format_dynamic_echo(s, d, material))
        for r in results:
            fh.write(format_results(r))


def dtester_errors(a: Results, b: Results) -> dict:
    """The metric of the reference's golden-file checker (src/dtester.c:204-262):
    max over rows of the row 1-norm of the difference; for the stresses the
    per-point max-row norms of the 3x3 tensors are summed over points."""
    def norm1(x, y):
        return float(np.max(np.sum(np.abs(x - y), axis=1))) if len(x) else 0.0

    sig = 0.0
    for p, q in zip(a.sigma, b.sigma):
        sig += norm1(p.reshape(3, 3), q.reshape(3, 3))
    return {"disp": norm1(a.disp, b.disp), "traction": norm1(a.traction, b.traction),
            "idisp": norm1(a.idisp, b.idisp), "sigma": sig}
