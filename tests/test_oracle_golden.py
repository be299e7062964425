"""Pins the CPU oracle against the reference's own known-answer tests.

src/tests.sh:38-117 runs ESOLO240 and ESOLO2160 and checks the dynamic output
with src/dtester.c (max row 1-norm of the difference <= EPS = 1e-3 for the
boundary displacements, tractions, interior displacements and stresses).
"""
import os

import numpy as np
import pytest

import oracle
from bem_mececcs_b200 import formats, host, meshgen

EPS = 1.0e-3  # src/dtester.c:24


def _run(golden_dir, tag):
    s = formats.read_static(os.path.join(golden_dir, f"ESOLO{tag}E_-5+5.DAT"))
    d = formats.read_dynamic(os.path.join(golden_dir, f"ESOLO{tag}D_-5+5.DAT"), s.nbe)
    p = oracle.OracleProblem(s, d)
    p.ghmatece()
    fr = d.freqs[0]
    disp, tr, _ = p.solve(fr)
    zdsol, zssol = p.interior(fr, disp, tr)
    mine = formats.Results(fr, disp.reshape(-1, 3), tr.reshape(-1, 3),
                           zdsol.reshape(-1, 3), zssol.reshape(-1, 9))
    gold = formats.parse_results(os.path.join(golden_dir, f"SSOLO{tag}D_-5+5.SOL"))
    assert len(gold) == 1 and gold[0].disp.shape == (s.nbe, 3)
    return mine, gold[0]


def test_oracle_matches_golden_240(golden_dir):
    mine, gold = _run(golden_dir, "240")
    err = formats.dtester_errors(mine, gold)
    assert all(np.isfinite(list(err.values())))
    assert all(v <= EPS for v in err.values()), err


@pytest.mark.slow
def test_oracle_matches_golden_2160(golden_dir):
    mine, gold = _run(golden_dir, "2160")
    err = formats.dtester_errors(mine, gold)
    assert all(v <= EPS for v in err.values()), err


def test_gauleg_matches_exact_rule():
    # Gauss-Legendre nodes/weights are known to double precision.
    for npg in (2, 4, 8):
        gi, ome = oracle.gauleg(npg)
        x, w = np.polynomial.legendre.leggauss(npg)
        assert np.allclose(gi, x, atol=1e-14) and np.allclose(ome, w, atol=1e-14)


def test_restated_zgesv_matches_lapack():
    rng = np.random.default_rng(7)
    n = 300
    a = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    b = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    x1 = oracle.zgesv(a, b, use_openblas=False)
    x2 = oracle.zgesv(a, b, use_openblas=True)
    assert np.linalg.norm(x1 - x2) / np.linalg.norm(x2) < 1e-12
    assert np.linalg.norm(a @ x1 - b) / np.linalg.norm(b) < 1e-12


def test_parser_roundtrip(tmp_path, golden_dir):
    s = formats.read_static(os.path.join(golden_dir, "ESOLO240E_-5+5.DAT"))
    d = formats.read_dynamic(os.path.join(golden_dir, "ESOLO240D_-5+5.DAT"), s.nbe)
    formats.write_static(tmp_path / "e.dat", s)
    formats.write_dynamic(tmp_path / "d.dat", d)
    s2 = formats.read_static(tmp_path / "e.dat")
    d2 = formats.read_dynamic(tmp_path / "d.dat", s2.nbe)
    assert (s2.n, s2.nbe, s2.np, s2.npg) == (s.n, s.nbe, s.np, s.npg)
    assert np.array_equal(s2.cone, s.cone) and np.array_equal(s2.cx, s.cx)
    assert np.array_equal(d2.kode, d.kode) and np.array_equal(d2.bc, d.bc)
    assert np.array_equal(d2.cxi, d.cxi) and d2.freqs.tolist() == d.freqs.tolist()


def test_results_format_roundtrip(tmp_path, golden_dir):
    gold = formats.parse_results(os.path.join(golden_dir, "SSOLO240D_-5+5.SOL"))[0]
    path = tmp_path / "out.sol"
    path.write_text(formats.format_results(gold), encoding="latin-1")
    back = formats.parse_results(path)[0]
    err = formats.dtester_errors(back, gold)
    assert max(err.values()) == 0.0


@pytest.mark.parametrize("tag", ["240", "2160"])
def test_static_echo_is_byte_exact(golden_dir, tag):
    """src/tests.sh:41-46: the static output (INPUTECE's echo with the element
    centroids the solver collocates at) equals the shipped SSOLO*E file byte
    for byte, from the reader and the centroids the product path uses."""
    s = formats.read_static(os.path.join(golden_dir, f"ESOLO{tag}E_-5+5.DAT"))
    with open(os.path.join(golden_dir, f"SSOLO{tag}E_-5+5.SOL"), encoding="latin-1") as fh:
        gold = fh.read()
    assert formats.format_static_echo(s) == gold


@pytest.mark.parametrize("tag", ["240", "2160"])
def test_dynamic_echo_is_byte_exact(golden_dir, tag):
    """The head of the shipped SSOLO*D file (INPUTECD's echo, with the derived
    complex material ZGE, ZCS, ZCP that the product path computes) byte for byte."""
    s = formats.read_static(os.path.join(golden_dir, f"ESOLO{tag}E_-5+5.DAT"))
    d = formats.read_dynamic(os.path.join(golden_dir, f"ESOLO{tag}D_-5+5.DAT"), s.nbe)
    with open(os.path.join(golden_dir, f"SSOLO{tag}D_-5+5.SOL"), encoding="latin-1") as fh:
        lines = fh.read().split("\n")
    i = next(k for k, ln in enumerate(lines) if "FREQ\xdc\xcaNCIA =" in ln)
    echo = formats.format_dynamic_echo(s, d, host.material(s.ge, s.rnu, d.dam, d.rho))
    assert echo == "\n".join(lines[:i - 3]) + "\n"


@pytest.mark.parametrize("tag", ["240", pytest.param("2160", marks=pytest.mark.slow)])
def test_oracle_output_file_is_the_shipped_one(tmp_path, golden_dir, tag):
    """src/tests.sh:48-53 at its strictest: the oracle's whole dynamic output
    file (echo + result block, 4 printed digits) IS SSOLO*D_-5+5.SOL."""
    s = formats.read_static(os.path.join(golden_dir, f"ESOLO{tag}E_-5+5.DAT"))
    d = formats.read_dynamic(os.path.join(golden_dir, f"ESOLO{tag}D_-5+5.DAT"), s.nbe)
    mine, _ = _run(golden_dir, tag)
    out = tmp_path / "out.sol"
    formats.write_dynamic_output(out, s, d, host.material(s.ge, s.rnu, d.dam, d.rho), [mine])
    with open(os.path.join(golden_dir, f"SSOLO{tag}D_-5+5.SOL"), "rb") as fh:
        assert out.read_bytes() == fh.read()


def test_fixtures_match_their_checksums(golden_dir):
    import hashlib
    with open(os.path.join(golden_dir, "SHA256SUMS")) as fh:
        sums = [ln.split() for ln in fh if ln.strip()]
    assert len(sums) == 12
    for digest, name in sums:
        with open(os.path.join(golden_dir, name), "rb") as fh:
            assert hashlib.sha256(fh.read()).hexdigest() == digest, name


@pytest.mark.parametrize("tag", ["240", "2160"])
def test_results_block_is_byte_exact(golden_dir, tag):
    """format_results re-creates the shipped result block (Outputec.for:21-59)
    byte for byte from the parsed values: labels, Fortran D formats, spacing."""
    path = os.path.join(golden_dir, f"SSOLO{tag}D_-5+5.SOL")
    lines = open(path, encoding="latin-1").read().split("\n")
    i = next(k for k, ln in enumerate(lines) if "FREQ\xdc\xcaNCIA =" in ln)
    block = "\n".join(lines[i - 3:])
    assert formats.format_results(formats.parse_results(path)[0]) == block


def test_oracle_static_solve_satisfies_its_system():
    """The static extension's restatement: H x = G dfi after the swap, and
    the prescribed values come back unchanged through the un-swap."""
    s, d = meshgen.config_mesh("c1_240")
    d.kode[::5] = 0
    d.bc[::5] = 0.02
    p = oracle.OracleProblem(s, d)
    disp, trac, h, g = p.static_solve(want_matrices=True)
    nn = 3 * s.nbe
    H = h.reshape(nn, nn, order="F")
    G = g.reshape(nn, nn, order="F")
    dfi = np.real(d.bc)
    x = np.where(d.kode == 0, trac / s.ge, disp)
    assert np.linalg.norm(H @ x - G @ dfi) < 1e-12 * np.linalg.norm(G @ dfi)
    k0 = d.kode == 0
    assert np.array_equal(disp[k0], dfi[k0]) and np.array_equal(trac[~k0], dfi[~k0])


def test_timing_build_computes_the_same_system(tmp_path):
    """The benchmark's CPU leg times bem_oracle.c built with the reference's
    flags (-march=native -Ofast ...); it must still compute GHMATECD, to the
    rounding that fast-math allows."""
    path, why = oracle.timing_lib(str(tmp_path))
    if path is None:
        pytest.skip(f"no compiler for the timing build: {why}")
    s, d = meshgen.config_mesh("c1_240")
    ref = oracle.OracleProblem(s, d)
    fast = oracle.OracleProblem(s, d, lib_path=path)
    assert fast._lib is not ref._lib
    zh0, zg0 = ref.ghmatecd(1.0)
    zh1, zg1 = fast.ghmatecd(1.0)
    assert np.linalg.norm(zh1 - zh0) <= 1e-11 * np.linalg.norm(zh0)
    assert np.linalg.norm(zg1 - zg0) <= 1e-11 * np.linalg.norm(zg0)


def test_oracle_reports_a_collapsed_element():
    """The GPU test's failure case, on the oracle: an element collapsed onto a
    line has DET < 1e-5, where the reference's CPU routines stop with
    'NONSING : ERRO, JACOBIANO NULO OU NEGATIVO' (src/Nonsinge.for:88,
    src/Nonsingd.for:89-94) and its GPU kernels return status 1 with 'Matriz
    Singular' (src/kernels/Ghmatecd_cu.cu:438); the oracle's static and
    dynamic assemblies both report status 1."""
    s, d = meshgen.config_mesh("c1_240")
    c = s.cone[5] - 1
    s.cx[c[2]], s.cy[c[2]] = s.cx[c[1]], s.cy[c[1]]
    s.cx[c[3]], s.cy[c[3]] = s.cx[c[0]], s.cy[c[0]]
    p = oracle.OracleProblem(s, d)
    with pytest.raises(RuntimeError, match="GHMATECE status 1"):
        p.ghmatece()
    p.hestdiag = np.zeros(9 * s.nbe)  # skip the static part to reach GHMATECD
    p.gestdiag = np.zeros(9 * s.nbe)
    with pytest.raises(RuntimeError, match="GHMATECD status 1"):
        p.ghmatecd(1.0)


@pytest.mark.parametrize("use_openblas", [False, True])
def test_oracle_zgesv_reports_a_singular_matrix(use_openblas):
    rng = np.random.default_rng(4)
    a = rng.standard_normal((40, 40)) + 1j * rng.standard_normal((40, 40))
    a[:, 17] = 0.0
    with pytest.raises(np.linalg.LinAlgError):
        oracle.zgesv(a, np.ones(40, dtype=np.complex128), use_openblas=use_openblas)


def test_smallest_enclosed_mesh_solves():
    """One boundary element (n = 3) in its enclosure: the smallest system."""
    s = meshgen.enclosed_grid(1, 1, jitter=0.0, seed=0, depth=2.5, layers=1)
    d = meshgen.traction_patch(s, radius=2.0, freqs=(1.0,))
    assert s.nbe == 1
    p = oracle.OracleProblem(s, d)
    p.ghmatece()
    zh, zfi, _, _ = p.system(1.0)
    disp, trac, x = p.solve(1.0, use_openblas=False)
    a = zh.reshape(3, 3, order="F")
    assert np.all(np.isfinite(x)) and np.linalg.norm(a @ x - zfi) <= 1e-13 * np.linalg.norm(zfi)


def test_parity_bound_resolves_small_physics_changes():
    """The 1e-10 relative bound the GPU is held to has teeth: a change of one
    part in 1e8 in the Poisson ratio or in omega moves the assembled system by
    8e-10 and 4.7e-9, so a device path computing a slightly different problem
    cannot pass it."""
    import copy
    s, d = meshgen.config_mesh("c1_240")

    def system(s1, fr):
        p = oracle.OracleProblem(s1, d)
        p.ghmatece()
        return p.system(fr)[0]

    zh0 = system(s, 1.0)
    s2 = copy.deepcopy(s)
    s2.rnu *= 1 + 1e-8
    for zh in (system(s2, 1.0), system(s, 1.0 + 1e-8)):
        assert np.linalg.norm(zh - zh0) / np.linalg.norm(zh0) > 5e-10
