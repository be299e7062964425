"""Fortran edit descriptors of the output writers (formats._fmt_d, _fmt_i)
and the writers at the large-mesh sizes where the reference's fixed-width
fields overflow."""
import numpy as np
import pytest

from bem_mececcs_b200 import formats, meshgen


@pytest.mark.parametrize("v,w,d,out", [
    (0.1, 11, 4, " 0.1000D+00"),
    (43.2, 11, 4, " 0.4320D+02"),
    (9.99996, 11, 4, " 0.1000D+02"),      # rounding carries into the exponent
    (-0.00012345, 11, 4, "-0.1234D-03"),  # 0.00012345 is below ...345 in binary
    (0.0, 10, 3, " 0.000D+00"),
    (5.0, 14, 7, " 0.5000000D+01"),
    (-5.0, 14, 7, "-0.5000000D+01"),
    (1e-120, 11, 4, " 0.1000-119"),       # three-digit exponent drops the D
    (1.0, 19, 7, "      0.1000000D+01"),
])
def test_d_descriptor(v, w, d, out):
    assert formats._fmt_d(v, w, d) == out


@pytest.mark.parametrize("v,w,out", [(7, 4, "   7"), (9999, 4, "9999"), (10000, 4, "****"),
                                     (-12, 4, " -12"), (-123, 3, "***"), (np.int32(240), 4, " 240")])
def test_i_descriptor(v, w, out):
    assert formats._fmt_i(v, w) == out


def test_large_mesh_echo_overflows_like_fortran():
    s = meshgen.enclosed_grid(110, 100, jitter=0.1, seed=0, depth=2.5, layers=1)
    assert s.n > 9999 and s.np > 9999
    lines = formats.format_static_echo(s).split("\n")
    assert "  N\xdaMERO DE ELEMENTOS DA MALHA= ****" in lines
    assert "  N\xdaMERO DE ELEMENTOS DE CONTORNO= ****" in lines  # nbe = 11000
    first = lines.index(f"    PONTO{'':10s}X{'':18s}Y{'':18s}Z") + 1
    assert lines[first + 9998].startswith("    9999") and lines[first + 9999].startswith("    ****")


def test_result_block_roundtrip_at_a_large_mesh(tmp_path):
    rng = np.random.default_rng(2)
    nbe = 12000
    c = lambda *sh: rng.standard_normal(sh) + 1j * rng.standard_normal(sh)  # noqa: E731
    r = formats.Results(2.5, c(nbe, 3), c(nbe, 3), np.zeros((0, 3)), np.zeros((0, 9)))
    p = tmp_path / "r.sol"
    p.write_text(formats.format_results(r), encoding="latin-1")
    back = formats.parse_results(p)[0]
    assert back.freq == 2.5 and back.disp.shape == (nbe, 3)
    # 4 printed digits: relative error of each part below 5e-4
    for a, b in ((back.disp, r.disp), (back.traction, r.traction)):
        for part in (np.real, np.imag):
            assert np.all(np.abs(part(a) - part(b)) <= 5e-4 * np.abs(part(b)) + 1e-300)


def test_truncated_input_file_is_reported(tmp_path, golden_dir):
    """A bad file fails on the host with the reader's error, before any device
    work: the static input cut in the middle of its connectivity, and the
    dynamic input cut in its boundary conditions."""
    import os
    src = open(os.path.join(golden_dir, "ESOLO240E_-5+5.DAT"), encoding="latin-1").read().split("\n")
    cut = tmp_path / "e.dat"
    cut.write_text("\n".join(src[: len(src) // 2]) + "\n", encoding="latin-1")
    with pytest.raises(EOFError, match="past the end"):
        formats.read_static(cut)
    s = formats.read_static(os.path.join(golden_dir, "ESOLO240E_-5+5.DAT"))
    dsrc = open(os.path.join(golden_dir, "ESOLO240D_-5+5.DAT"), encoding="latin-1").read().split("\n")
    dcut = tmp_path / "d.dat"
    dcut.write_text("\n".join(dsrc[:20]) + "\n", encoding="latin-1")
    with pytest.raises(EOFError):
        formats.read_dynamic(dcut, s.nbe)


def test_non_numeric_field_is_reported(tmp_path, golden_dir):
    import os
    src = open(os.path.join(golden_dir, "ESOLO240E_-5+5.DAT"), encoding="latin-1").read().split("\n")
    i = next(k for k in range(1, len(src)) if src[k].strip())  # the N, NBE, NP, NPG, GE, RNU record
    src[i] = src[i].replace(src[i].split()[0], "24O", 1)      # a letter O for a zero
    bad = tmp_path / "e.dat"
    bad.write_text("\n".join(src), encoding="latin-1")
    with pytest.raises(ValueError):
        formats.read_static(bad)
